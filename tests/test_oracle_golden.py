"""Pin the FP64 oracle to the reference's own golden values (CPU only).

Sources (reference paths): the golden CSVs of
FoggySim/ground_truth/lib_math_vector_spherical_harmonics and the inline values of the Fortran
unit tests, extracted into tests/golden by tests/golden/make_fixtures.py.
"""
import csv
import math
import os

import numpy as np
import pytest
from scipy.special import spherical_jn, spherical_yn

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_wigner_3j_table5(oracle, golden):
    g = golden["wigner_3j"]
    for j3, ref in zip(g["j3"], g["values"]):
        v = oracle.wigner_3j(g["j1"], g["j2"], j3, g["m1"], g["m2"], g["m3"])
        assert abs(v - ref) <= g["tol"], (j3, v, ref)


def test_ab_xu_cruzan(oracle, golden):
    # lib_math_vector_spherical_harmonics.f90:2799-2875
    g = golden["ab_xu_cruzan"]
    for q, ga, gb in zip(g["q"], g["a"], g["b"]):
        p = g["n"] + g["nu"] - 2 * q
        a, b = oracle.ab_xu_cruzan(g["m"], g["n"], g["mu"], g["nu"], p)
        assert abs(a - ga) <= g["tol"] and abs(b - gb) <= g["tol"], (q, a, ga, b, gb)


def test_spherical_bessel_j_x5(oracle, golden):
    g = golden["sph_jn_x5"]
    vals = oracle.sph_jn(g["x"], len(g["values"]) - 1)
    rel = np.abs(vals - np.array(g["values"])) / np.abs(g["values"])
    assert rel.max() <= g["tol"], rel.max()


def test_riccati_xi_x05(oracle, golden):
    # xi_n(x) = x h_n^(1)(x) = x j_n + i x y_n
    g = golden["riccati_xi_x05"]
    n = len(g["re"]) - 1
    x = g["x"]
    re = x * oracle.sph_jn(x, n)
    im = x * oracle.sph_yn(x, n)
    assert np.max(np.abs(1 - np.abs(re / np.array(g["re"])))) <= g["tol"]
    assert np.max(np.abs(1 - np.abs(im / np.array(g["im"])))) <= g["tol"]


@pytest.mark.parametrize("x", [0.3, 2.0, 5.712, 11.4, 37.0, 250.0, 790.0])
def test_spherical_bessel_vs_scipy(oracle, x):
    n = 70
    j = oracle.sph_jn(x, n)
    y = oracle.sph_yn(x, n)
    jr = spherical_jn(np.arange(n + 1), x)
    yr = spherical_yn(np.arange(n + 1), x)
    big = np.abs(jr) > 1e-280
    assert np.max(np.abs(j[big] - jr[big]) / np.maximum(np.abs(jr[big]), 1e-300)) < 1e-11
    fin = np.isfinite(yr)
    assert np.max(np.abs(y[fin] - yr[fin]) / np.abs(yr[fin])) < 1e-11


def test_pi_tau_theta2(oracle, golden):
    g = golden["pi_tau_theta2"]
    nmax = g["n_max"]
    pi, tau = oracle.pi_tau(g["theta"], nmax, cs_phase=True)
    for key, ref in g["pi"].items():
        n, m = map(int, key.split(","))
        assert abs(pi[n * (n + 1) + m] - ref) <= g["tol_pi"], (n, m, pi[n * (n + 1) + m], ref)
    for key, ref in g["tau"].items():
        n, m = map(int, key.split(","))
        assert abs(tau[n * (n + 1) + m] - ref) <= g["tol_tau"], (n, m, tau[n * (n + 1) + m], ref)


def test_pi_tau_phase_removed_for_odd_m(oracle):
    pi_cs, tau_cs = oracle.pi_tau(0.7, 6, cs_phase=True)
    pi, tau = oracle.pi_tau(0.7, 6, cs_phase=False)
    for n in range(1, 7):
        for m in range(-n, n + 1):
            s = -1 if abs(m) % 2 else 1
            assert pi[n * (n + 1) + m] == pytest.approx(s * pi_cs[n * (n + 1) + m], rel=1e-15, abs=0)


@pytest.mark.parametrize("theta", [0.0, math.pi])
def test_pi_tau_poles_are_limits(oracle, theta):
    # The reference's special pole values (lib_math_legendre.f90:854-920) equal the limits of
    # the general formula, except tau_n^{-1} for odd n at theta = pi, whose sign the reference
    # flips (it copies -pi_n^{-1} there); the oracle keeps that.
    pi0, tau0 = oracle.pi_tau(theta, 8)
    eps = 1e-7
    pi1, tau1 = oracle.pi_tau(theta + eps if theta == 0 else theta - eps, 8)
    if theta != 0:
        for n in range(1, 9, 2):
            tau1[n * (n + 1) - 1] = -tau1[n * (n + 1) - 1]
    assert np.max(np.abs(pi0 - pi1)) < 1e-4 * np.max(np.abs(pi0))
    assert np.max(np.abs(tau0 - tau1)) < 1e-4 * np.max(np.abs(tau0))


def test_mie_ab_barber_hill(oracle, golden):
    g = golden["mie_ab_m15_x10"]
    a, b = oracle.mie_ab(g["x"], g["m"], 1, 4)
    for i in range(4):
        ga = complex(*g["a"][i])
        gb = complex(*g["b"][i])
        assert abs(a[i] / ga - 1) <= g["tol"], (i, a[i], ga)
        assert abs(b[i] / gb - 1) <= g["tol"], (i, b[i], gb)


def _read_ab(fn):
    rows = []
    with open(os.path.join(GOLD, fn)) as f:
        r = csv.reader(f)
        next(r)
        for row in r:
            m, n, mu, nu = (int(float(v)) for v in row[:4])
            rows.append((m, n, mu, nu, complex(float(row[4]), float(row[5])), complex(float(row[6]), float(row[7]))))
    return rows


@pytest.mark.parametrize("fn,phi", [("ground_truth_AB_mnmunu.csv", 0.5),
                                    ("ground_truth_AB_mnmunu_minus_phi.csv", 2 * math.pi - 0.5)])
def test_translation_coefficients_golden(oracle, fn, phi):
    # lib_math_vector_spherical_harmonics.f90:2876-3168: x = 2, theta = 0.5, z = 3, n, nu <= 5
    A, B = oracle.translation_xu(2.0, 0.5, phi, (1, 5), (1, 5), 3)
    worst = 0.0
    for m, n, mu, nu, ga, gb in _read_ab(fn):
        r = n * n - 1 + n + m
        c = nu * nu - 1 + nu + mu
        for v, ref in ((A[r, c], ga), (B[r, c], gb)):
            if ref == 0:
                assert abs(v) < 1e-13
            else:
                worst = max(worst, abs(v - ref) / abs(ref))
    assert worst < 1e-12, worst


def test_universal_index_golden(oracle, golden):
    for case in golden["universal_index"]:
        assert oracle.universal_index(np.array(case["point"]), case["l"]) == case["n"]


def test_coordinate_binary_bits(oracle):
    # 0.75 -> 0b11 followed by zeros in the 64-bit fraction; 0 -> 0
    assert oracle.coordinate_binary(0.75) == (3 << 62)
    assert oracle.coordinate_binary(0.5) == (1 << 63)
    assert oracle.coordinate_binary(0.0) == 0
    x = 0.3
    assert oracle.coordinate_binary(x) >> 11 == int(x * 2 ** 53)


def test_single_sphere_extinction_matches_mie_formula(oracle):
    # one sphere: the cluster formula reduces to Q_ext = 2/x^2 sum (2n+1) Re(a_n + b_n)
    from itofoggysim_b200 import scene as S
    sc = S.make_scene(np.array([0.5]), 1.0, 0, z_coupling=3)
    P = oracle.Problem(sc)
    b = P.vector_b()
    cs = P.cross_sections(b)
    x = sc.wavenumber * 0.5
    a, bb = oracle.mie_ab(x, S.M_WATER, 1, sc.n_range[1])
    qext = 2 / x ** 2 * np.sum((2 * np.arange(1, len(a) + 1) + 1) * np.real(a + bb))
    assert cs[1] / (math.pi * 0.25) == pytest.approx(qext, rel=1e-12)
    assert cs[0] + cs[2] == pytest.approx(cs[1], rel=1e-14)
