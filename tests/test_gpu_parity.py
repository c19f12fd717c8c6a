"""Parity of the CUDA path (through the C ABI) with the FP64 oracle.

Error metric for coefficient vectors: the reference layout stores x_nm, whose size scales with
g_nm = sqrt((n+m)!/(n-m)!); vectors are compared after dividing by g_nm (the basis the device
works in), as max |x - x_ref| / max |x_ref|.  Tolerances: 1e-12 for single operator
applications, 1e-10 for converged solves (both solved to <= 1e-13).
"""
import math

import numpy as np
import pytest

from itofoggysim_b200 import _native, scene as S, solver

pytestmark = pytest.mark.gpu


def g_of_layout(sc):
    pg = sc.n_range[1]
    g = []
    for n in range(1, pg + 1):
        for m in range(-n, n + 1):
            g.append(math.sqrt(math.factorial(n + m) / math.factorial(n - m)))
    g = np.array(g)
    return np.tile(np.concatenate([g, g]), sc.n_spheres)


def scaled_err(x, ref, sc):
    g = g_of_layout(sc)
    a, r = x / g, ref / g
    return np.max(np.abs(a - r)) / max(np.max(np.abs(r)), 1e-300)


def random_scaled(sc, seed):
    rng = np.random.default_rng(seed)
    n = sc.vector_length()
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    x *= g_of_layout(sc)
    # entries above a sphere's own degree are zero in a solution vector
    pg = sc.n_range[1]
    C = (pg + 1) ** 2 - 1
    p = sc.p_of_sphere()
    xv = x.reshape(sc.n_spheres, 2, C)
    for j in range(sc.n_spheres):
        xv[j, :, p[j] * (p[j] + 2):] = 0
    return x


WAVES = {
    "z_tm": S.single_wave(),
    "oblique_mixed": S.single_wave(0.7, 1.1, (0.6, 0.0, 0.0, 0.3)),
    "minus_z": S.single_wave(math.pi, 0.3, (0.2, 0.1, 0.9, -0.4)),
    "two_waves": dict(wave_theta=np.array([0.3, 2.0]), wave_phi=np.array([0.0, -1.0]),
                      jones=np.array([[1.0, 0.0, 0.0, 0.0], [0.0, 0.0, 1.0, 0.0]]),
                      wave_g=np.array([1.0, 0.5]), wave_phase=np.array([0.0, 0.4]),
                      wave_d0=np.array([[0.0, 0.0, 0.0], [0.3, -0.2, 1.0]])),
}


def test_mie_coefficients(native, oracle):
    sc = S.random_cluster(5, seed=11, p=None)
    P = oracle.Problem(sc)
    with solver.MultiSphereSolver(sc) as s:
        for ip in range(sc.n_param):
            a, b = s.mie_coefficients(ip)
            ra, rb = P.mie(ip)
            p = len(a)
            assert np.max(np.abs(a - ra[:p]) / np.abs(ra[:p])) < 1e-12
            assert np.max(np.abs(b - rb[:p]) / np.abs(rb[:p])) < 1e-12


def test_mie_coefficients_golden(native, golden):
    # m = 1.5, x = 10 (lib_mie_ss_helper_functions.f90:1639-1703), through a one-sphere scene
    g = golden["mie_ab_m15_x10"]
    lam = 0.55
    r = g["x"] * lam / (2 * math.pi)
    sc = S.make_scene(np.array([r]), 1.0, 0, m=complex(g["m"], 0.0), n_max=4)
    with solver.MultiSphereSolver(sc) as s:
        a, b = s.mie_coefficients(0)
    for i in range(4):
        assert abs(a[i] / complex(*g["a"][i]) - 1) <= g["tol"]
        assert abs(b[i] / complex(*g["b"][i]) - 1) <= g["tol"]


@pytest.mark.parametrize("wave", sorted(WAVES))
def test_vector_b(native, oracle, wave):
    sc = S.random_cluster(6, seed=3, waves=WAVES[wave])
    P = oracle.Problem(sc)
    with solver.MultiSphereSolver(sc) as s:
        b = s.get_vector_b()
    assert scaled_err(b, P.vector_b(), sc) < 1e-12


@pytest.mark.parametrize("z", [1, 3])
@pytest.mark.parametrize("case", range(4))
def test_translation_coefficients(native, oracle, z, case):
    rng = np.random.default_rng(100 + case)
    x = rng.uniform(2.0, 40.0)
    th = [0.0, math.pi, rng.uniform(0, math.pi), 1e-9][case]
    ph = rng.uniform(-math.pi, math.pi)
    pn, pnu = [(5, 5), (7, 4), (10, 10), (3, 9)][case]
    A, B = solver.translation_coefficient(x, th, ph, (1, pn), (1, pnu), z)
    Ao, Bo = oracle.translation_xu(x, th, ph, (1, pn), (1, pnu), z)
    gn = np.array([math.sqrt(math.factorial(n + m) / math.factorial(n - m)) for n in range(1, pn + 1)
                   for m in range(-n, n + 1)])
    gnu = np.array([math.sqrt(math.factorial(n + m) / math.factorial(n - m)) for n in range(1, pnu + 1)
                    for m in range(-n, n + 1)])
    for M, Mo in ((A, Ao), (B, Bo)):
        Ms = M / gn[:, None] * gnu[None, :]
        Mos = Mo / gn[:, None] * gnu[None, :]
        assert np.max(np.abs(Ms - Mos)) <= 1e-12 * np.max(np.abs(Mos))


def test_translation_coefficients_golden(native):
    import csv
    import os
    # the golden entries span many decades through g_nm / g_nu,mu: compare in the scaled basis,
    # relative to the largest scaled entry (exact zeros of the table included)
    fn = os.path.join(os.path.dirname(__file__), "golden", "ground_truth_AB_mnmunu.csv")
    A, B = solver.translation_coefficient(2.0, 0.5, 0.5, (1, 5), (1, 5), 3)
    g = np.array([math.sqrt(math.factorial(n + m) / math.factorial(n - m)) for n in range(1, 6)
                  for m in range(-n, n + 1)])
    GA = np.zeros_like(A)
    GB = np.zeros_like(B)
    with open(fn) as f:
        r = csv.reader(f)
        next(r)
        for row in r:
            m, n, mu, nu = (int(float(v)) for v in row[:4])
            i, j = n * n - 1 + n + m, nu * nu - 1 + nu + mu
            GA[i, j] = complex(float(row[4]), float(row[5]))
            GB[i, j] = complex(float(row[6]), float(row[7]))
    for M, G in ((A, GA), (B, GB)):
        Ms = M / g[:, None] * g[None, :]
        Gs = G / g[:, None] * g[None, :]
        assert np.max(np.abs(Ms - Gs)) <= 1e-12 * np.max(np.abs(Gs))


MATVEC_CASES = [
    # n, p (None: per-sphere Wiscombe), z, reference_row_rule, seed
    (2, 4, 1, True, 1),
    (2, 4, 3, True, 2),
    (5, 6, 3, False, 3),
    (6, None, 3, False, 4),
    (6, None, 1, True, 5),
    (8, 3, 1, False, 6),
]


@pytest.mark.parametrize("pair_tables", [0, -1])
@pytest.mark.parametrize("n,p,z,rule,seed", MATVEC_CASES)
def test_matvec(native, oracle, n, p, z, rule, seed, pair_tables):
    # pair_tables 0: per-pair scalar coefficients kept in device memory; -1: rebuilt per call
    sc = S.random_cluster(n, seed=seed, p=p, z_coupling=z, reference_row_rule=rule)
    P = oracle.Problem(sc)
    x = random_scaled(sc, seed)
    with solver.MultiSphereSolver(sc, pair_tables=pair_tables) as s:
        y = s.calculate_vector_b(x)
        y2 = s.calculate_vector_b(x)
    yo = P.matvec(x)
    assert scaled_err(y, yo, sc) < 1e-12
    assert np.array_equal(y, y2), "operator is not bit-reproducible"


def test_matvec_identity_rows_above_own_degree(native, oracle):
    # entries above a sphere's degree pass through unchanged, as in the reference's y = x + ...
    sc = S.random_cluster(4, seed=9, p=None, reference_row_rule=False)
    rng = np.random.default_rng(0)
    x = (rng.standard_normal(sc.vector_length()) + 1j) * g_of_layout(sc)
    with solver.MultiSphereSolver(sc) as s:
        y = s.calculate_vector_b(x)
    pg = sc.n_range[1]
    C = (pg + 1) ** 2 - 1
    p = sc.p_of_sphere()
    for j in range(sc.n_spheres):
        P = p[j] * (p[j] + 2)
        blk = slice(2 * C * j, 2 * C * (j + 1))
        yj, xj = y[blk].reshape(2, C), x[blk].reshape(2, C)
        assert np.array_equal(yj[:, P:], xj[:, P:])


def test_single_sphere_is_identity(native):
    sc = S.random_cluster(1, seed=1, p=5)
    x = random_scaled(sc, 1)
    with solver.MultiSphereSolver(sc) as s:
        y = s.calculate_vector_b(x)
        b = s.get_vector_b()
        xs, st = s.solve()
    # identity up to the rounding of the x / g_nm -> g_nm x layout round trip
    assert scaled_err(y, x, sc) < 1e-15
    assert scaled_err(xs, b, sc) < 1e-15


@pytest.mark.parametrize("z", [1, 3])
def test_solve_vs_dense(native, oracle, z):
    sc = S.random_cluster(4, seed=21, p=4, z_coupling=z, reference_row_rule=True)
    sc.gmres_tolerance = 1e-14
    sc.gmres_restart = 40
    P = oracle.Problem(sc)
    n = P.n
    g = g_of_layout(sc)
    cols = []
    for i in range(n):
        e = np.zeros(n, np.complex128)
        e[i] = g[i]
        cols.append(P.matvec(e) / g)
    A = np.stack(cols, axis=1)
    b = P.vector_b()
    xs = np.linalg.solve(A, b / g) * g
    with solver.MultiSphereSolver(sc) as s:
        x, st = s.solve()
    assert st["status"] == 0 and st["backward_error"] <= 1e-14
    assert scaled_err(x, xs, sc) < 1e-10
    # the oracle's own GMRES (the reference's method) agrees as well
    xo, sto = P.solve(restart=40, tol=1e-14, weights=1.0 / g ** 2)
    assert scaled_err(xo, xs, sc) < 1e-10


def test_solve_initial_guess_and_cross_sections(native, oracle):
    sc = S.random_cluster(6, seed=5, p=None, z_coupling=3)
    sc.gmres_tolerance = 1e-13
    P = oracle.Problem(sc)
    g = g_of_layout(sc)
    with solver.MultiSphereSolver(sc, init_with_single_sphere=True) as s:
        x, st = s.solve()
        cs = s.cross_sections(x)
        # residual with the device operator
        r = s.get_vector_b() - s.calculate_vector_b(x)
    assert np.linalg.norm(r / g) / np.linalg.norm(P.vector_b() / g) < 1e-12
    xo, sto = P.solve(restart=30, tol=1e-13, weights=1.0 / g ** 2)
    assert scaled_err(x, xo, sc) < 1e-10
    # C_abs is ~1e-8 of C_ext for m = 1.33 + 1e-8 i and carries the cancellation of
    # Re(1/a_n) - 1: it is compared with an absolute tolerance relative to C_ext
    co = P.cross_sections(x)
    assert np.allclose(cs, co, rtol=1e-12, atol=1e-12 * co[1])
    cso = P.cross_sections(xo)
    assert np.allclose(cs, cso, rtol=1e-10, atol=1e-10 * cso[1])


def test_nan_input_reports_status(native):
    sc = S.random_cluster(3, seed=2, p=3)
    x0 = np.zeros(sc.vector_length(), np.complex128)
    x0[0] = np.nan
    with solver.MultiSphereSolver(sc) as s:
        x, st = s.solve(x0=x0, raise_on_error=False)
    assert st["status"] == _native.FOGGY_ERR_NAN


def test_not_converged_status(native):
    sc = S.random_cluster(6, seed=8, p=5, z_coupling=3)
    sc.gmres_tolerance = 1e-15
    sc.gmres_max_iterations = 3
    with solver.MultiSphereSolver(sc) as s:
        x, st = s.solve(raise_on_error=False)
    assert st["status"] == _native.FOGGY_ERR_NOT_CONVERGED and st["iterations"] == 3


def test_argument_errors(native):
    sc = S.random_cluster(3, seed=2, p=3)
    sc.param_index = np.array([0, 5, 0], np.int32)
    with pytest.raises(_native.FoggyError) as e:
        solver.MultiSphereSolver(sc)
    assert e.value.code == _native.FOGGY_ERR_ARGUMENT


def test_refused_scene_keeps_previous(native):
    """A foggy_set_spheres call refused for its input leaves the handle's scene as it was."""
    import ctypes as C
    sc = S.random_cluster(3, seed=2, p=3)
    with solver.MultiSphereSolver(sc) as s:
        b0 = s.get_vector_b()
        x0, _ = s.solve()
        c, pi, m, r, nr = s._keep
        bad = [np.array([0, 5, 0], np.int32), np.array([0, -1, 0], np.int32)]
        for pidx in bad:
            rc = s.L.foggy_set_spheres(s.h, sc.n_spheres, _native.ptr(c), _native.ptr(pidx, C.c_int32), sc.n_param,
                                       _native.ptr(m), _native.ptr(r), _native.ptr(nr, C.c_int32))
            assert rc == _native.FOGGY_ERR_ARGUMENT
        cen = c.copy()
        cen[4] = np.inf
        rc = s.L.foggy_set_spheres(s.h, sc.n_spheres, _native.ptr(cen), _native.ptr(pi, C.c_int32), sc.n_param,
                                   _native.ptr(m), _native.ptr(r), _native.ptr(nr, C.c_int32))
        assert rc == _native.FOGGY_ERR_ARGUMENT
        assert s.L.foggy_vector_length(s.h) == sc.vector_length()
        assert np.array_equal(s.get_vector_b(), b0)
        x1, st = s.solve()
        assert st["status"] == 0 and np.array_equal(x1, x0)


def test_memory_budget_admission(native):
    sc = S.random_cluster(6, seed=2, p=6)
    with pytest.raises(_native.FoggyError) as e:
        solver.MultiSphereSolver(sc, memory_budget=1000)
    assert e.value.code == _native.FOGGY_ERR_NOMEM


# ---- octree ------------------------------------------------------------------------------
def test_universal_index_golden(native, golden):
    for case in golden["universal_index"]:
        assert solver.universal_index(np.array([case["point"]]), case["l"])[0] == case["n"]


@pytest.mark.parametrize("level", [1, 3, 7, 21])
def test_universal_index_bit_exact(native, oracle, level):
    rng = np.random.default_rng(level)
    pts = rng.random((4000, 3))
    pts[:10] = [[0, 0, 0], [0.5, 0.5, 0.5], [1 - 2 ** -53, 0, 0.25], [2 ** -30, 2 ** -60, 0.75],
                [0.125, 0.999, 0.001], [0.3, 0.3, 0.3], [0.7, 0.1, 0.9], [2 ** -1022, 0.5, 0.5],
                [0.0, 1 - 2 ** -40, 0.0], [0.1, 0.2, 0.3]]
    u = solver.universal_index(pts, level)
    ref = np.array([oracle.universal_index(p, level) for p in pts])
    assert np.array_equal(u, ref)


@pytest.mark.parametrize("which", ["small", "random", "medium"])
def test_build_tree_matches_oracle(native, oracle, which):
    if which == "small":
        sc = S.small_cluster()
    elif which == "random":
        sc = S.random_cluster(300, seed=7, p=2)
        sc.tree_l_max = 0
    else:
        sc = S.medium_cluster()
    with solver.MultiSphereSolver(sc) as s:
        u, order, lmin, lmax = s.build_tree()
        uo, oo, lmino, lmaxo = oracle.build_tree(sc.centres, s=10, l_max=sc.tree_l_max)
        assert (lmin, lmax) == (lmino, lmaxo)
        assert np.array_equal(order, oo)
        assert np.array_equal(u, uo)
        for l in range(1, lmax + 1):
            boxes = s.tree_boxes(l)
            ref = np.unique(uo >> (3 * (lmaxo - l)))
            assert np.array_equal(boxes, ref)


# ---- the small-cluster workload at full size -------------------------------------------------
def test_small_cluster_full_size(native, oracle):
    """64 spheres, p = 15: GPU solve to 1e-8, its residual through the device operator, and the
    operator rows of one target sphere against the oracle (63 exact Xu translations)."""
    sc = S.small_cluster()
    P = oracle.Problem(sc)
    g = g_of_layout(sc)
    with solver.MultiSphereSolver(sc) as s:
        x, st = s.solve()
        assert st["status"] == 0 and st["backward_error"] <= 1e-8
        y = s.calculate_vector_b(x)
        b = s.get_vector_b()
    assert np.linalg.norm((b - y) / g) / np.linalg.norm(b / g) <= 1.01e-8
    assert scaled_err(b, P.vector_b(), sc) < 1e-12
    C = (sc.n_range[1] + 1) ** 2 - 1
    yo = P.pairs_apply(x, [0] * (sc.n_spheres - 1), list(range(1, sc.n_spheres))) + x
    blk = slice(0, 2 * C)
    gb = g[blk]
    assert np.max(np.abs((y[blk] - yo[blk]) / gb)) <= 1e-12 * np.max(np.abs(yo[blk] / gb))
