"""Physical checks of the oracle's multi-sphere solve, where the reference stores no solution to
compare with (CPU): a cluster of non-absorbing spheres absorbs nothing (C_ext = C_sca, which
checks the cluster cross-section formulas), widely separated spheres decouple, the coupling
falling as 1/(kd) with the outgoing spherical waves, and the translation coefficients have the
parity of a reversed displacement."""
import numpy as np

from itofoggysim_b200 import scene as S


def test_real_index_cluster_absorbs_nothing(oracle):
    sc = S.random_cluster(3, seed=4, p=5, z_coupling=3, m=complex(1.33, 0.0))
    P = oracle.Problem(sc)
    x, _ = P.solve(restart=30, tol=1e-13)
    c_sca, c_ext, c_abs = P.cross_sections(x)
    assert c_ext > 0 and abs(c_ext - c_sca) <= 1e-12 * c_ext and abs(c_abs) <= 1e-12 * c_ext


def test_absorbing_cluster_absorbs(oracle):
    sc = S.random_cluster(3, seed=4, p=5, z_coupling=3, m=complex(1.33, 0.05))
    P = oracle.Problem(sc)
    x, _ = P.solve(restart=30, tol=1e-13)
    c_sca, c_ext, c_abs = P.cross_sections(x)
    # C_abs comes from the absorption of each sphere's own field (Re(1/a_n) - 1 terms), not as a
    # difference; it is positive and below C_ext
    assert 1e-3 * c_ext < c_abs < c_ext and c_sca > 0


def coupling(oracle, distance):
    sc = S.random_cluster(2, seed=5, p=5, z_coupling=3)
    if distance is not None:
        sc.centres = np.array([[0.0, 0.0, 0.0], [0.0, 0.0, distance]])
    P = oracle.Problem(sc)
    b = P.vector_b()
    x, _ = P.solve(restart=30, tol=1e-14)
    return np.linalg.norm(x - b) / np.linalg.norm(b)


def test_separated_spheres_decouple_as_one_over_kd(oracle):
    near = coupling(oracle, None)
    far = [coupling(oracle, d) for d in (2000.0, 4000.0, 8000.0)]
    assert near > 0.05 and far[0] < 1e-3
    assert abs(far[0] / far[1] - 2.0) < 1e-3 and abs(far[1] / far[2] - 2.0) < 1e-3


def test_translation_parity(oracle):
    """Reversing the displacement (theta -> pi - theta, phi -> phi + pi) multiplies A by
    (-1)^(n + nu) and B by -(-1)^(n + nu), for regular and outgoing radial functions alike: the
    symmetry behind the reciprocity of a two-sphere system."""
    x, th, ph = 7.3, 0.7, 1.1
    n = np.array([n for n in range(1, 6) for m in range(-n, n + 1)])
    sgn = (-1.0) ** (n[:, None] + n[None, :])
    for z in (1, 3):
        A, B = oracle.translation_xu(x, th, ph, (1, 5), (1, 5), z)
        A2, B2 = oracle.translation_xu(x, np.pi - th, ph + np.pi, (1, 5), (1, 5), z)
        assert np.max(np.abs(A2 - sgn * A)) <= 1e-13 * np.max(np.abs(A))
        assert np.max(np.abs(B2 + sgn * B)) <= 1e-13 * np.max(np.abs(B))
