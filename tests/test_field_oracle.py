"""Vector spherical wave functions of the oracle against the reference's golden tables
(FoggySim/ground_truth/lib_math_vector_spherical_harmonics/ground_truth_M_mn.csv, _N_mn.csv:
theta = 0.2, phi = 0, k = 2 pi, r = 50, h_n^(1), n = 1..4; consumed at
libmath/src/math/lib_math_vector_spherical_harmonics.f90:2443-2575 with an absolute tolerance of
1e-13 on each spherical vector)."""
import math
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("which", ["M", "N"])
def test_vswf_matches_reference(oracle, which):
    M, N = oracle.vswf(0.2, 0.0, 50.0, 2.0 * math.pi, 4, 3)
    got = M if which == "M" else N
    rows = np.genfromtxt(os.path.join(HERE, "golden", "ground_truth_%s_mn.csv" % which),
                         delimiter=",", skip_header=1)
    assert len(rows) == 24
    for row in rows:
        n, m = int(row[0]), int(row[1])
        ref = np.array([row[2] + 1j * row[3], row[4] + 1j * row[5], row[6] + 1j * row[7]])
        assert np.linalg.norm(got[n * n - 1 + n + m] - ref) < 1e-13


def test_field_zero_inside_and_finite_outside(oracle):
    """The cluster's field is zero inside a sphere (lib_mie_ss_get_field returns zero for r <= radius,
    lib_mie_single_sphere.f90:1427-1433) and finite elsewhere."""
    from itofoggysim_b200 import scene as S
    sc = S.small_cluster()
    P = oracle.Problem(sc)
    rng = np.random.default_rng(5)
    x = rng.standard_normal(sc.vector_length()) + 1j * rng.standard_normal(sc.vector_length())
    c0 = np.asarray(sc.centres[0])
    r0 = float(sc.radius[sc.param_index[0]])
    pts = np.array([c0, c0 + np.array([0.0, 0.0, 4.0 * r0])])
    E, H = P.field(x, pts)
    assert np.all(E[0] == 0) and np.all(H[0] == 0)
    assert np.all(np.isfinite(E[1])) and np.max(np.abs(E[1])) > 0
