"""Gaussian beams in the plane-wave approximation (the reference's calculation_type 3,
FoggySim/src/lib/mie_theory/lib_mie_illumination.f90:781-918, 1022-1050;
FoggySim/src/lib/field/lib_field_gaussian_beam.f90) in the oracle, checked with the reference's
own tests (lib_field_gaussian_beam.f90:922-1210, 1570-1684: the scalar field equals
|E| exp(i arg E) on a grid for TEM11 in both conventions, and the local plane wave reproduces the
beam's field on the axis; tolerance 1e-7 as there) and with properties of the beam."""
import math

import numpy as np
import pytest
from numpy.polynomial import hermite as npH

from itofoggysim_b200 import fields

UM = 1.0   # lengths in micrometres


@pytest.mark.parametrize("convention", [1, 2])
def test_scalar_equals_abs_arg(oracle, convention):
    xs = np.arange(-10.0, 10.0, 1.0)
    pts = np.array([[x, y, 10.0] for x in xs for y in xs])
    s, aa, _ = oracle.gaussian_probe(0.55, 1.0, (2.0, 2.0), (1, 1), (1, 0, 0, 0), 0.0, 0.0, 0.0, convention, pts)
    rebuilt = aa[:, 0] * np.exp(1j * aa[:, 1])
    assert np.max(np.abs(s - rebuilt)) < 1e-7
    assert np.max(np.abs(s - rebuilt)) < 1e-12 * max(1.0, np.max(np.abs(s)))
    assert np.all((aa[:, 1] >= 0) & (aa[:, 1] < 2 * math.pi))


def test_plane_wave_approximation_on_axis(oracle):
    pts = np.array([[0.0, 0.0, 5.0]])
    s, aa, wv = oracle.gaussian_probe(0.5, 1.0, (2.5, 2.5), (0, 0), (1, 0, 0, 0), 0.0, 0.0, 0.0, 1, pts)
    th, ph, jxr, jxi, jyr, jyi, phase, amp = wv[0]
    assert th == 0.0 and abs(amp - aa[0, 0]) < 1e-15
    E_pw, _ = fields.plane_wave_field(pts, 0.5, 1.0, th, ph, (complex(jxr, jxi), complex(jyr, jyi)),
                                      e_field_0=amp, phase=phase)
    E_g = s[0] * np.array([1.0, 0.0, 0.0])
    assert np.max(np.abs(E_pw[0] - E_g)) < 1e-7


def test_direction_diverges_and_polarisation_is_unit(oracle):
    pts = np.array([[1.0, 0.0, 8.0], [-1.0, 0.5, 8.0], [1.0, 0.0, -8.0], [0.0, 0.0, 3.0]])
    jones = (math.cos(0.3), 0.0, math.sin(0.3), 0.2)
    _, _, wv = oracle.gaussian_probe(0.55, 1.33, (1.5, 1.5), (0, 0), jones, 0.0, 0.0, 0.4, 1, pts)
    k = np.stack([np.sin(wv[:, 0]) * np.cos(wv[:, 1]), np.sin(wv[:, 0]) * np.sin(wv[:, 1]), np.cos(wv[:, 0])], 1)
    assert k[0, 0] > 0 and k[1, 0] < 0 and k[2, 0] < 0      # away from the axis after the waist
    assert np.all(k[:, 2] > 0.9) and wv[3, 0] == 0.0       # forward, on axis exactly along z
    pol = np.abs(wv[:, 2] + 1j * wv[:, 3]) ** 2 + np.abs(wv[:, 4] + 1j * wv[:, 5]) ** 2
    assert np.allclose(pol, 1.0, atol=1e-14)


def test_rotated_beam_direction(oracle):
    # a beam tilted to theta = 0.6, phi = 1.1 propagates along that direction on its axis
    th, ph = 0.6, 1.1
    d = np.array([math.sin(th) * math.cos(ph), math.sin(th) * math.sin(ph), math.cos(th)])
    _, _, wv = oracle.gaussian_probe(0.55, 1.0, (2.0, 2.0), (0, 0), (1, 0, 0, 0), th, ph, 0.0, 1, 5.0 * d[None, :])
    k = np.array([math.sin(wv[0, 0]) * math.cos(wv[0, 1]), math.sin(wv[0, 0]) * math.sin(wv[0, 1]), math.cos(wv[0, 0])])
    assert np.allclose(k, d, atol=1e-12)


def test_hermite_against_numpy(oracle):
    # H_n through the scalar field's x factor: Hermite-Gauss TEM_m0 at z = 0 with w0 = sqrt(2)
    # gives sqrt(1/(2^m m! pi)) H_m(x) exp(-x^2/2)
    for m in range(0, 7):
        xs = np.linspace(-2.5, 2.5, 11)
        pts = np.stack([xs, 0 * xs, 0 * xs], 1)
        s, _, _ = oracle.gaussian_probe(0.55, 1.0, (math.sqrt(2.0), math.sqrt(2.0)), (m, 0), (1, 0, 0, 0),
                                        0.0, 0.0, 0.0, 1, pts)
        c = np.zeros(m + 1)
        c[m] = 1.0
        ref = npH.hermval(xs, c) * np.exp(-xs ** 2 / 2) * math.sqrt(1.0 / (2 ** m * math.factorial(m) * math.pi))
        ref = ref * np.exp(1j * 0.5 * 0.0)   # Gouy phase 0 at z = 0
        assert np.max(np.abs(s - ref)) < 1e-12 * max(1.0, np.max(np.abs(ref)))


def test_beam_rhs_in_oracle(oracle):
    """The oracle's right-hand side with one Gaussian beam is the plane-wave right-hand side of each
    sphere's local plane wave, scaled by g twice."""
    from itofoggysim_b200 import scene as S
    sc = S.random_cluster(4, seed=2, p=4)
    P = oracle.Problem(sc)
    b_pw = P.vector_b()
    P.set_gaussian_beams((3.0, 3.0), (0, 0), [0.0], [0.0], (1, 0, 0, 0), [0.5], [0.0], [0.0, 0.0, -4.0])
    b_all = P.vector_b()
    C = (sc.n_range[1] + 1) ** 2 - 1
    for j in range(sc.n_spheres):
        xw = sc.centres[j] - np.array([0.0, 0.0, -4.0])
        _, _, wv = oracle.gaussian_probe(sc.lambda_0, sc.n_medium, (3.0, 3.0), (0, 0), (1, 0, 0, 0), 0.0, 0.0,
                                         0.0, 1, xw[None, :])
        th, ph, jxr, jxi, jyr, jyi, phase, _ = wv[0]
        one = S.Scene(**{**sc.__dict__, "centres": sc.centres[j:j + 1], "param_index": sc.param_index[j:j + 1],
                         "wave_theta": np.array([th]), "wave_phi": np.array([ph]),
                         "jones": np.array([[jxr, jxi, jyr, jyi]]), "wave_g": np.array([0.25]),
                         "wave_phase": np.array([phase]), "wave_d0": np.array([[0.0, 0.0, -4.0]])})
        bj = oracle.Problem(one).vector_b()
        got = (b_all - b_pw)[2 * C * j:2 * C * (j + 1)]
        assert np.max(np.abs(got - bj)) <= 1e-13 * max(1e-300, np.max(np.abs(bj)))
