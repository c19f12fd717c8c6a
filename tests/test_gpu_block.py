"""Several right-hand sides in one block: the block operator and the batched GMRES solve.

The block operator (foggy_matvec_block) applies the direct operator to many vectors at once, a tile
of them per CTA; it must equal foggy_matvec (pinned to the oracle by test_gpu_parity.py and
test_gpu_high_order.py) vector by vector: 1e-13 in FP64 (the sums over sources run in another
order), 1e-5 with FP32 translation arithmetic.  The block solve (foggy_solve_block) must give each
right-hand side the solution of its own solve (foggy_solve_rhs): 1e-10 in FP64 with both solved to
1e-12, 1e-6 in mixed precision, for 128 right-hand sides (64 Fibonacci
directions x TM/TE) of the 64-sphere cluster.

Error metric: vectors divided by g_nm (the basis the device works in), max |x - ref| / max |ref|.
"""
import dataclasses
import math

import numpy as np
import pytest

from itofoggysim_b200 import scene as S, solver

pytestmark = pytest.mark.gpu


def _g_layout(sc):
    g = np.array([math.sqrt(math.factorial(n + m) / math.factorial(n - m))
                  for n in range(1, sc.n_range[1] + 1) for m in range(-n, n + 1)])
    return np.tile(np.concatenate([g, g]), sc.n_spheres)


def _err(x, ref, g):
    a, r = x / g, ref / g
    return np.max(np.abs(a - r)) / max(np.max(np.abs(r)), 1e-300)


def _vectors(sc, nv, seed):
    rng = np.random.default_rng(seed)
    g = _g_layout(sc)
    n = sc.vector_length()
    X = (rng.standard_normal((nv, n)) + 1j * rng.standard_normal((nv, n))) * g
    C = (sc.n_range[1] + 1) ** 2 - 1
    p = sc.p_of_sphere()
    Xv = X.reshape(nv, sc.n_spheres, 2, C)
    for j in range(sc.n_spheres):
        Xv[:, j, :, p[j] * (p[j] + 2):] = 0
    return X


def fibonacci_waves(n_dir):
    """64 directions on a Fibonacci sphere (z_i = 1 - (2i+1)/n, phi_i = i pi (3 - sqrt 5)) x TM, TE."""
    i = np.arange(n_dir)
    th = np.arccos(1.0 - (2.0 * i + 1.0) / n_dir)
    ph = np.mod(i * math.pi * (3.0 - math.sqrt(5.0)), 2.0 * math.pi)
    n = 2 * n_dir
    return dict(wave_theta=np.repeat(th, 2), wave_phi=np.repeat(ph, 2),
                jones=np.tile([[1.0, 0.0, 0.0, 0.0], [0.0, 0.0, 1.0, 0.0]], (n_dir, 1)),
                wave_g=np.ones(n), wave_phase=np.zeros(n), wave_d0=np.zeros((n, 3)))


SCENES = {
    # mixed orders 3..15 (several buckets), z = h_n, reference row rule off
    "mixed": lambda: S.random_cluster(12, seed=31, p=None, z_coupling=3, reference_row_rule=False),
    # the reference's own settings: z = j_n, coupling rows zeroed below the global order
    "reference_rule": lambda: S.random_cluster(9, seed=32, p=None, z_coupling=1, reference_row_rule=True),
    # orders 17..30 (the upper buckets of the lognormal benchmark scene)
    "high_order": lambda: S.random_cluster(6, seed=41, radii=np.array([0.6, 0.7, 0.95, 1.15, 1.3, 1.5]), box=8.0,
                                           z_coupling=3, reference_row_rule=False),
}


@pytest.mark.parametrize("pair_tables", [0, -1])
@pytest.mark.parametrize("case", sorted(SCENES))
def test_block_matvec_matches_single(native, case, pair_tables):
    sc = SCENES[case]()
    g = _g_layout(sc)
    nv = 11   # not a multiple of any tile width: the last tile is partial
    X = _vectors(sc, nv, 5)
    with solver.MultiSphereSolver(sc, pair_tables=pair_tables) as s:
        Y1 = np.stack([s.calculate_vector_b(x) for x in X])
        Yb = s.calculate_vector_b_block(X, precision=0)
        Yb2 = s.calculate_vector_b_block(X, precision=0)
        Yf = s.calculate_vector_b_block(X, precision=1)
        tiles = s.block_tiles(nv, precision=0)
    assert np.array_equal(Yb, Yb2), "block operator is not bit-reproducible"
    for v in range(nv):
        assert _err(Yb[v], Y1[v], g) < 1e-13, "vector %d" % v
        assert _err(Yf[v], Y1[v], g) < 1e-5, "vector %d (FP32)" % v
    assert set(tiles[:, 3].tolist()) <= {1, 2, 4, 8}
    assert np.all(tiles[:, 0] > 0) and np.all(tiles[:, 2] <= 32)


def test_block_matvec_one_vector(native):
    sc = SCENES["mixed"]()
    g = _g_layout(sc)
    X = _vectors(sc, 1, 9)
    with solver.MultiSphereSolver(sc) as s:
        y1 = s.calculate_vector_b(X[0])
        yb = s.calculate_vector_b_block(X)[0]
    assert _err(yb, y1, g) < 1e-13


@pytest.fixture(scope="module")
def cluster_128():
    sc = S.small_cluster()
    return dataclasses.replace(sc, **fibonacci_waves(64), gmres_tolerance=1e-12, name="small_cluster_64_rhs128")


@pytest.fixture(scope="module")
def solo_128(native, cluster_128):
    with solver.MultiSphereSolver(cluster_128) as s:
        x, cs, st = s.solve_rhs()
    return x, cs


def test_block_solve_fp64_matches_solo(native, cluster_128, solo_128):
    sc = cluster_128
    g = _g_layout(sc)
    xs, css = solo_128
    with solver.MultiSphereSolver(sc) as s:
        x, cs, its, be, st = s.solve_block()
    assert st["status"] == 0
    assert np.all(be <= 1e-12) and np.all(its > 0)
    assert st["iterations"] == int(its.sum())
    for r in range(sc.n_waves):
        assert _err(x[r], xs[r], g) < 1e-10, "right-hand side %d" % r
    assert np.allclose(cs[:, 1], css[:, 1], rtol=1e-10, atol=0)


def test_block_solve_mixed_matches_solo(native, cluster_128, solo_128):
    sc = dataclasses.replace(cluster_128, gmres_tolerance=1e-8)
    g = _g_layout(sc)
    xs, css = solo_128
    with solver.MultiSphereSolver(sc, precision=1) as s:
        x, cs, its, be, st = s.solve_block()
    assert st["status"] == 0
    assert np.all(be <= 1e-8)
    for r in range(sc.n_waves):
        rel = np.linalg.norm((x[r] - xs[r]) / g) / np.linalg.norm(xs[r] / g)
        assert rel < 1e-6, "right-hand side %d: %.2e" % (r, rel)
    assert np.allclose(cs[:, 1], css[:, 1], rtol=1e-6, atol=0)


def test_block_solve_with_initial_guess_and_limits(native):
    sc = S.random_cluster(8, seed=33, p=None, z_coupling=3)
    sc = dataclasses.replace(sc, **fibonacci_waves(3), gmres_tolerance=1e-11, gmres_restart=5)
    g = _g_layout(sc)
    with solver.MultiSphereSolver(sc) as s:
        xs, _, _ = s.solve_rhs()
        # started from the solutions: every right-hand side leaves the block at the first residual
        x, _, its, be, st = s.solve_block(x0=xs)
        assert st["status"] == 0 and np.all(its == 0)
        for r in range(sc.n_waves):
            assert _err(x[r], xs[r], g) < 1e-14
        # an iteration limit below what the tolerance needs is reported per right-hand side
        s.set_max_iterations(2)
        x, _, its, be, st = s.solve_block(raise_on_error=False)
        assert st["status"] == -5 and np.all(its <= 2) and np.all(be > 1e-11)


def test_block_solve_through_the_mlfmm(native):
    """A block over the ML-FMM operator (consistent passes, boxes small against the wavelength; its
    passes run vector after vector inside each block application): each right-hand side within 1e-10
    of its own ML-FMM solve, FP64 and mixed precision (1e-6)."""
    rng = np.random.default_rng(7)
    sc = S.make_scene(rng.uniform(0.1, 0.3, 30), 9.0, 5, lambda_0=6.0, n_max=6, z_coupling=3,
                      reference_row_rule=False, tree_l_max=3, waves=fibonacci_waves(3), gmres_tolerance=1e-12)
    g = _g_layout(sc)
    with solver.MultiSphereSolver(sc, use_ml_fmm=True, fmm_convention=1) as s:
        xs, _, _ = s.solve_rhs()
        x, cs, its, be, st = s.solve_block()
        assert st["status"] == 0 and np.all(be <= 1e-12)
        for r in range(sc.n_waves):
            assert _err(x[r], xs[r], g) < 1e-10, "right-hand side %d" % r
    sc2 = dataclasses.replace(sc, gmres_tolerance=1e-8)
    with solver.MultiSphereSolver(sc2, use_ml_fmm=True, fmm_convention=1, precision=1) as s:
        x32, _, _, be32, st32 = s.solve_block()
    assert st32["status"] == 0 and np.all(be32 <= 1e-8)
    for r in range(sc.n_waves):
        assert np.linalg.norm((x32[r] - xs[r]) / g) <= 1e-6 * np.linalg.norm(xs[r] / g)


def test_block_argument_errors(native):
    """Refusals of the block entries: right-hand-side count other than the plane waves set, an
    unknown precision."""
    import ctypes as C
    from itofoggysim_b200 import _native as N
    sc = S.random_cluster(4, seed=34, p=3)
    sc = dataclasses.replace(sc, **fibonacci_waves(2))
    n = sc.vector_length()
    x = np.zeros(4 * n, np.complex128)
    st = N.FoggyStats()
    with solver.MultiSphereSolver(sc) as s:
        assert s.L.foggy_solve_block(s.h, 3, None, x.ctypes.data, N.FOGGY_MEM_HOST, C.byref(st), None, None,
                                     None) == N.FOGGY_ERR_ARGUMENT
        assert s.L.foggy_matvec_block(s.h, 2, 2, x.ctypes.data, x.ctypes.data, N.FOGGY_MEM_HOST) == N.FOGGY_ERR_ARGUMENT
        xs, cs, its, be, st2 = s.solve_block()
        assert st2["status"] == 0 and xs.shape == (4, n)
