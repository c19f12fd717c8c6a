"""Several right-hand sides: the operator applied to 2, 3, 4 and 7 vectors per call
(foggy_matvec_rhs) equals foggy_matvec of each vector bit for bit, with and without pair tables,
and foggy_solve_rhs returns for each plane wave what foggy_solve returns for that wave alone, with
and without the single-sphere initial guess."""
import numpy as np
import pytest

from itofoggysim_b200 import scene as S, solver

pytestmark = pytest.mark.gpu


def _waves(rng, n):
    th = np.arccos(rng.uniform(-1, 1, n))
    ph = rng.uniform(0, 2 * np.pi, n)
    jo = np.where((np.arange(n) % 2 == 0)[:, None], [[1.0, 0.0, 0.0, 0.0]], [[0.0, 0.0, 1.0, 0.0]])
    return dict(wave_theta=th, wave_phi=ph, jones=jo, wave_g=np.ones(n), wave_phase=np.zeros(n),
                wave_d0=np.zeros((n, 3)))


@pytest.mark.parametrize("nv", [2, 3, 4, 7])
@pytest.mark.parametrize("tables", [0, -1])
def test_batched_operator_equals_single(native, nv, tables):
    sc = S.random_cluster(9, seed=5, p=None, z_coupling=3)
    rng = np.random.default_rng(nv)
    with solver.MultiSphereSolver(sc, pair_tables=tables) as s:
        X = (rng.standard_normal((nv, s.n)) + 1j * rng.standard_normal((nv, s.n))) * 1e-3
        Y = s.calculate_vector_b_rhs(X)
        for v in range(nv):
            assert np.array_equal(Y[v], s.calculate_vector_b(X[v]))


@pytest.mark.parametrize("guess", [False, True])
def test_rhs_solves_equal_single_solves(native, guess):
    rng = np.random.default_rng(11)
    sc = S.random_cluster(10, seed=8, p=6, waves=_waves(rng, 6))
    with solver.MultiSphereSolver(sc, init_with_single_sphere=guess) as s:
        xs, css, st = s.solve_rhs()
    assert st["backward_error"] <= sc.gmres_tolerance
    keys = ("wave_theta", "wave_phi", "jones", "wave_g", "wave_phase", "wave_d0")
    for r in range(sc.n_waves):
        one = S.Scene(**{**sc.__dict__, **{k: getattr(sc, k)[r:r + 1] for k in keys}})
        with solver.MultiSphereSolver(one, init_with_single_sphere=guess) as s1:
            x1, st1 = s1.solve()
            c1 = s1.cross_sections(x1)
        assert np.array_equal(xs[r], x1)
        assert np.array_equal(css[r], c1)
