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


def _fmm_lists(s):
    import ctypes as C
    from itofoggysim_b200 import _native
    parts = []
    for part in range(12):
        cnt = C.c_int32(0)
        _native.check(s.L.foggy_fmm_lists(s.h, part, None, C.byref(cnt)), s.h)
        out = np.zeros(max(cnt.value, 1), np.int32)
        _native.check(s.L.foggy_fmm_lists(s.h, part, _native.ptr(out, C.c_int32), C.byref(cnt)), s.h)
        parts.append(out[:cnt.value])
    return parts


def _csr(lists):
    ptr = np.concatenate([[0], np.cumsum([len(v) for v in lists])]).astype(np.int32)
    idx = np.array([i for v in lists for i in v], np.int32)
    return ptr, idx


@pytest.mark.parametrize("n,lmax,rule", [(40, 3, False), (300, 4, False), (24, 2, True), (1, 3, False)])
def test_device_fmm_lists_match_oracle(native, oracle, n, lmax, rule):
    """The ML-FMM's pass lists, built on the device from the sorted keys, against the lists that
    follow from the oracle's hierarchy and domains (E1, E2, I4 of the reference's libtree)."""
    sc = S.random_cluster(n, seed=50 + n, p=None if rule else 3, reference_row_rule=rule)
    sc.tree_l_max = lmax
    with solver.MultiSphereSolver(sc, use_ml_fmm=True) as s:
        u, order, lmin, lmax_ = s.build_tree()
        got = _fmm_lists(s)
    assert lmax_ == lmax
    uo, oo, lmino, lmaxo = oracle.build_tree(sc.centres, s=10, l_max=lmax)
    lmin = min(lmino, lmax)
    boxes = {l: np.unique(uo >> (3 * (lmax - l))) for l in range(lmin, lmax + 1)}
    gid, base = {}, 0
    for l in range(lmin, lmax + 1):
        for k, b in enumerate(boxes[l]):
            gid[(l, int(b))] = base + k
        base += len(boxes[l])
    leaves = [int(b) for b in boxes[lmax]]
    p = sc.p_of_sphere()
    couple = np.ones(n, bool) if not rule else (p >= sc.n_range[1])
    e1 = {b: oracle.tree_domain(sc.centres, lmax, lmax, b, 1) for b in leaves}
    e2 = {b: oracle.tree_domain(sc.centres, lmax, lmax, b, 2) for b in leaves}
    leaf_of = {int(j): gid[(lmax, b)] for b in leaves for j in e1[b]}
    ref = []
    ref += _csr([[int(j) for j in e1[b] if couple[j]] for b in leaves])
    kids, i4, par = [], [], []
    for l in range(lmin, lmax + 1):
        for b in boxes[l]:
            b = int(b)
            kids.append([gid[(l + 1, int(c))] for c in boxes.get(l + 1, []) if int(c) >> 3 == b])
            cand = oracle.tree_domain(sc.centres, lmax, l, b, 4)
            i4.append([gid[(l, int(c))] for c in cand if (l, int(c)) in gid])
            par.append([gid[(l - 1, b >> 3)]] if l > lmin else [])
    ref += _csr(kids) + _csr(i4) + _csr(par)
    ref += _csr([[leaf_of[j]] for j in range(n)])
    leaf_box = {gid[(lmax, b)]: b for b in leaves}
    ref += _csr([[int(i) for i in e2[leaf_box[leaf_of[j]]] if i != j] for j in range(n)])
    names = ["aggregation ptr", "aggregation idx", "children ptr", "children idx", "I4 ptr", "I4 idx",
             "parent ptr", "parent idx", "box-to-sphere ptr", "box-to-sphere idx", "near ptr", "near idx"]
    for k in range(12):
        assert np.array_equal(got[k], ref[k]), names[k]


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


@pytest.mark.parametrize("n,p,z,conv,rule,lmax", CASES)
def test_fmm_tables_equal_gaunt_sums(native, n, p, z, conv, rule, lmax):
    """The passes' cached coaxial blocks (one per distinct translation length and degrees of each
    pass list) against S summed from the Gaunt table per translation (pair_tables = -1): the same
    operator bit for bit, in both conventions (the reference's shifted box-to-sphere step
    included), and the same again after the radial function changes (the blocks are rebuilt)."""
    sc = S.random_cluster(n, seed=n + (p or 0), p=p, z_coupling=z, reference_row_rule=rule)
    sc.tree_l_max = lmax
    x = _x(sc, 4)
    out = {}
    for pt in (0, -1):
        with solver.MultiSphereSolver(sc, use_ml_fmm=True, fmm_convention=conv, z_translation_gt_r=3,
                                      pair_tables=pt) as s:
            y1 = s.calculate_vector_b(x)
            s.params.z_coupling = 4 if z != 4 else 3
            s._set()
            y2 = s.calculate_vector_b(x)
        out[pt] = (y1, y2)
    assert np.array_equal(out[0][0], out[-1][0])
    assert np.array_equal(out[0][1], out[-1][1])
    assert not np.array_equal(out[0][0], out[0][1])


LEVEL_CASES = [
    # n, p, convention, digits (boxes of an 8 um cube at lambda = 6 um: per-level orders 5..9)
    (16, 3, 1, 2.0),
    (16, 3, 0, 2.0),
    (20, 4, 1, 1.0),
]


@pytest.mark.parametrize("n,p,conv,digits", LEVEL_CASES)
def test_per_level_orders_match_oracle(native, oracle, n, p, conv, digits):
    """Boxes expanded to per-level orders (fmm_digits > 0: the excess-bandwidth order of the level's
    box diagonal, never below the global order): the device passes against the oracle's restatement
    at 1e-12, with the cached translation blocks bit-identical to the per-translation sums."""
    sc = long_wave_scene(p, n=n)
    x = _x(sc, 6)
    ref = oracle.Problem(sc).fmm_matvec(x, l_max=3, convention=conv, z_gt_r=3, digits=digits)
    ys = []
    for pt in (0, -1):
        with solver.MultiSphereSolver(sc, use_ml_fmm=True, fmm_convention=conv, z_translation_gt_r=3,
                                      pair_tables=pt, fmm_digits=digits) as s:
            ys.append(s.calculate_vector_b(x))
    assert _err(ys[0], ref, _g(sc)) < 1e-12
    assert np.array_equal(ys[0], ys[1])
    with solver.MultiSphereSolver(sc, use_ml_fmm=True, fmm_convention=conv, z_translation_gt_r=3) as s:
        y_global = s.calculate_vector_b(x)
    assert not np.array_equal(y_global, ys[0])


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
