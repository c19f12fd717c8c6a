"""Parity of the CUDA operator with the FP64 oracle at truncation orders 17-30, and up to the
reference's cap of 45.

The 2000-sphere lognormal scene (radii 0.2-1.5 um at lambda = 0.55 um) has per-sphere Wiscombe
orders up to 30, median 17.  These tests cover those degrees, every truncation-order bucket of
the operator (17-20, 21-24, 25-28, 29-32), both radial functions of the coupling and both ways of
getting the scalar coaxial coefficients (pair tables kept in device memory, or summed from the
Gaunt table per application):

  * whole operator applications on a 6-sphere scene with orders 17..30 (1e-12, scaled basis);
  * operator rows of high-order targets on the full 2000-sphere scene, with a source vector that
    is zero except on a few spheres, so the oracle only needs those pairs (1e-12);
  * the single-pair translation coefficients A, B at n, nu up to 30 (1e-12);
  * the FP32 operator of the mixed-precision solve at these orders: its solution against the
    FP64 solution (1e-6 relative) with the FP64 backward error reached.

Error metric: vectors divided by g_nm = sqrt((n+m)!/(n-m)!) (the basis the device works in),
max |x - x_ref| / max |x_ref|, as in test_gpu_parity.py.
"""
import math

import numpy as np
import pytest

from itofoggysim_b200 import scene as S, solver

pytestmark = pytest.mark.gpu

TOL_OP = 1e-12
TOL_MIXED = 1e-6

# radii whose Wiscombe orders at lambda = 0.55 um are 17, 18, 22, 25, 27, 30 (checked below)
HIGH_RADII = np.array([0.6, 0.7, 0.95, 1.15, 1.3, 1.5])
HIGH_P = [17, 18, 22, 25, 27, 30]

_oracle_cache = {}


def _g_layout(sc):
    g = np.array([math.sqrt(math.factorial(n + m) / math.factorial(n - m))
                  for n in range(1, sc.n_range[1] + 1) for m in range(-n, n + 1)])
    return np.tile(np.concatenate([g, g]), sc.n_spheres)


def _scaled_err(x, ref, g):
    a, r = x / g, ref / g
    return np.max(np.abs(a - r)) / max(np.max(np.abs(r)), 1e-300)


def _random_scaled(sc, seed, g, support=None):
    """Random vector of O(1) scaled entries, zero above each sphere's order and, with support,
    zero outside those spheres."""
    rng = np.random.default_rng(seed)
    n = sc.vector_length()
    x = (rng.standard_normal(n) + 1j * rng.standard_normal(n)) * g
    C = (sc.n_range[1] + 1) ** 2 - 1
    p = sc.p_of_sphere()
    xv = x.reshape(sc.n_spheres, 2, C)
    for j in range(sc.n_spheres):
        xv[j, :, p[j] * (p[j] + 2):] = 0
        if support is not None and j not in support:
            xv[j] = 0
    return x


def high_order_scene(z):
    return S.random_cluster(6, seed=41, radii=HIGH_RADII, box=8.0, z_coupling=z, reference_row_rule=False)


def _oracle_matvec(oracle, z):
    if z not in _oracle_cache:
        sc = high_order_scene(z)
        g = _g_layout(sc)
        x = _random_scaled(sc, 7, g)
        _oracle_cache[z] = (x, oracle.Problem(sc).matvec(x))
    return _oracle_cache[z]


def test_high_order_scene_orders():
    sc = high_order_scene(3)
    p = sc.p_of_sphere()
    assert sorted(p.tolist()) == HIGH_P
    # one sphere in each truncation-order bucket of the operator launches
    assert {(int(v) - 1) // 4 for v in p} == {4, 5, 6, 7}


@pytest.mark.parametrize("pair_tables", [0, -1])
@pytest.mark.parametrize("z", [1, 3])
def test_matvec_orders_17_to_30(native, oracle, z, pair_tables):
    sc = high_order_scene(z)
    g = _g_layout(sc)
    x, yo = _oracle_matvec(oracle, z)
    with solver.MultiSphereSolver(sc, pair_tables=pair_tables) as s:
        y = s.calculate_vector_b(x)
        y2 = s.calculate_vector_b(x)
    assert _scaled_err(y, yo, g) < TOL_OP
    assert np.array_equal(y, y2), "operator is not bit-reproducible"
    # every target sphere's rows on their own (the largest-order spheres dominate the max norm)
    C = (sc.n_range[1] + 1) ** 2 - 1
    for j in range(sc.n_spheres):
        blk = slice(2 * C * j, 2 * C * (j + 1))
        assert _scaled_err(y[blk], yo[blk], g[blk]) < TOL_OP, "sphere %d (p = %d)" % (j, sc.p_of_sphere()[j])


def test_medium_cluster_rows_at_full_size(native, oracle):
    """The 2000-sphere lognormal scene as the benchmark runs it (all buckets, all launches, the
    pair tables when they fit): x is zero except on five source spheres, so the rows of a target
    are x_j + T_j sum over those five pairs, which the oracle computes exactly."""
    sc = S.medium_cluster()
    p = sc.p_of_sphere()
    order = np.argsort(p, kind="stable")
    # sources: the two highest orders, the median and the two lowest; targets: the highest order,
    # a sphere of order 24-28, the median, the lowest
    src = [int(order[-1]), int(order[-2]), int(order[len(order) // 2]), int(order[0]), int(order[1])]
    mid = [int(j) for j in order if 24 <= p[j] <= 28 and int(j) not in src][:1]
    tgt = [int(order[-3]), int(order[len(order) // 2 + 1]), int(order[2])] + mid + [src[0]]
    assert max(p[tgt]) == 30 or max(p[src]) == 30
    g = _g_layout(sc)
    x = _random_scaled(sc, 11, g, support=set(src))
    P = oracle.Problem(sc)
    pj, pl = [], []
    for j in tgt:
        for l in src:
            if l != j:
                pj.append(j)
                pl.append(l)
    yo = P.pairs_apply(x, pj, pl) + x
    with solver.MultiSphereSolver(sc) as s:
        y = s.calculate_vector_b(x)
    C = (sc.n_range[1] + 1) ** 2 - 1
    for j in tgt:
        blk = slice(2 * C * j, 2 * C * (j + 1))
        assert _scaled_err(y[blk], yo[blk], g[blk]) < TOL_OP, "target %d (p = %d)" % (j, p[j])


@pytest.mark.parametrize("z", [1, 3])
@pytest.mark.parametrize("pn,pnu,x,th", [(30, 30, 31.0, 0.9), (30, 17, 23.5, 2.3), (22, 27, 40.0, 1e-9)])
def test_translation_coefficients_orders_to_30(native, oracle, z, pn, pnu, x, th):
    ph = -1.3
    A, B = solver.translation_coefficient(x, th, ph, (1, pn), (1, pnu), z)
    Ao, Bo = oracle.translation_xu(x, th, ph, (1, pn), (1, pnu), z)
    gn = np.array([math.sqrt(math.factorial(n + m) / math.factorial(n - m)) for n in range(1, pn + 1)
                   for m in range(-n, n + 1)])
    gnu = np.array([math.sqrt(math.factorial(n + m) / math.factorial(n - m)) for n in range(1, pnu + 1)
                    for m in range(-n, n + 1)])
    for M, Mo in ((A, Ao), (B, Bo)):
        Ms = M / gn[:, None] * gnu[None, :]
        Mos = Mo / gn[:, None] * gnu[None, :]
        assert np.max(np.abs(Ms - Mos)) <= TOL_OP * np.max(np.abs(Mos))


@pytest.mark.parametrize("pair_tables", [0, -1])
def test_mixed_precision_orders_17_to_30(native, pair_tables):
    """FP32 operator (single-precision pair tables, d(pi/2) table and coaxial sums) in the Arnoldi
    steps, FP64 true residual at each restart: the solution meets the FP64 tolerance and agrees
    with the FP64 solve, whose operator the tests above pin to the oracle."""
    sc = high_order_scene(3)
    sc.gmres_tolerance = 1e-10
    g = _g_layout(sc)
    with solver.MultiSphereSolver(sc, pair_tables=pair_tables) as s:
        x64, st64 = s.solve()
    with solver.MultiSphereSolver(sc, pair_tables=pair_tables, precision=1) as s:
        x32, st32 = s.solve()
        r = s.get_vector_b() - s.calculate_vector_b(x32)
        b = s.get_vector_b()
    assert st64["status"] == 0 and st32["status"] == 0
    assert st32["backward_error"] <= 1e-10
    assert np.linalg.norm(r / g) / np.linalg.norm(b / g) <= 1.01e-10
    rel = np.linalg.norm((x32 - x64) / g) / np.linalg.norm(x64 / g)
    assert rel < TOL_MIXED


def test_matvec_orders_33_to_45(native, oracle):
    """Spheres above order 32 (radius 1.8 and 2.6 um at 0.55 um: orders 34 and 45, the reference's cap,
    lib_mie_ss_helper_functions.f90:32): they fall in the operator's upper order buckets (33-36,
    45-48), whose CTAs use up to 216 KB of shared memory."""
    sc = S.random_cluster(2, seed=43, radii=np.array([1.8, 2.6]), box=8.0, z_coupling=3,
                          reference_row_rule=False)
    assert sorted(sc.p_of_sphere().tolist()) == [34, 45]
    g = _g_layout(sc)
    x = _random_scaled(sc, 8, g)
    yo = oracle.Problem(sc).matvec(x)
    for pair_tables in (0, -1):
        with solver.MultiSphereSolver(sc, pair_tables=pair_tables) as s:
            y = s.calculate_vector_b(x)
            yb = s.calculate_vector_b_block(np.stack([x, x]), precision=0)
        assert _scaled_err(y, yo, g) < TOL_OP, pair_tables
        assert _scaled_err(yb[1], yo, g) < TOL_OP, pair_tables

