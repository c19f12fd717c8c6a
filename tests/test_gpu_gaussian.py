"""Gaussian-beam right-hand side on the device (foggy_set_gaussian_beams) against the oracle's
restatement of the reference's plane-wave approximation (lib_mie_illumination.f90:781-918 case 3,
lib_field_gaussian_beam.f90:256-358), alone and added to plane waves, at 1e-12 of the largest
entry; and a solve driven by a beam alone."""
import numpy as np
import pytest

from itofoggysim_b200 import scene as S, solver

pytestmark = pytest.mark.gpu

BEAMS = {
    "tem00_axis": dict(waist=[[2.0, 2.0]], tem=[[0, 0]], theta=[0.0], phi=[0.0], jones=[[1, 0, 0, 0]], g=[0.7],
                       phase=[0.0], d_0_i=[[0.0, 0.0, -5.0]], convention=[1]),
    "tilted_tem11": dict(waist=[[1.6, 2.4]], tem=[[1, 1]], theta=[0.5], phi=[1.2],
                         jones=[[0.6, 0.1, 0.3, -0.7]], g=[1.0], phase=[0.3], d_0_i=[[0.4, -0.2, -3.0]],
                         convention=[2]),
    "two_beams": dict(waist=[[2.0, 2.0], [3.0, 1.5]], tem=[[0, 0], [2, 0]], theta=[0.0, 2.6], phi=[0.0, -0.8],
                      jones=[[1, 0, 0, 0], [0, 0, 1, 0]], g=[0.5, 0.9], phase=[0.0, 1.0],
                      d_0_i=[[0.0, 0.0, -5.0], [1.0, 1.0, 4.0]], convention=[1, 1]),
}


def _rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("case", sorted(BEAMS))
@pytest.mark.parametrize("with_plane_wave", [True, False])
def test_beam_rhs_matches_oracle(native, oracle, case, with_plane_wave):
    sc = S.random_cluster(6, seed=3, p=5)
    bm = BEAMS[case]
    P = oracle.Problem(sc)
    with solver.MultiSphereSolver(sc) as s:
        if not with_plane_wave:
            s.set_plane_waves([], [], np.zeros((0, 4)), [], [], np.zeros((0, 3)))
            sc0 = S.Scene(**{**sc.__dict__, "wave_theta": np.zeros(0), "wave_phi": np.zeros(0),
                             "jones": np.zeros((0, 4)), "wave_g": np.zeros(0), "wave_phase": np.zeros(0),
                             "wave_d0": np.zeros((0, 3))})
            P = oracle.Problem(sc0)
        s.set_gaussian_beams(**bm)
        P.set_gaussian_beams(bm["waist"], bm["tem"], bm["theta"], bm["phi"], bm["jones"], bm["g"], bm["phase"],
                             bm["d_0_i"], bm["convention"])
        b = s.get_vector_b()
    bo = P.vector_b()
    assert np.max(np.abs(bo)) > 0
    assert _rel(b, bo) < 1e-12


def test_solve_with_beam_only(native, oracle):
    sc = S.random_cluster(6, seed=3, p=5)
    with solver.MultiSphereSolver(sc) as s:
        s.set_plane_waves([], [], np.zeros((0, 4)), [], [], np.zeros((0, 3)))
        s.set_gaussian_beams(**BEAMS["tem00_axis"])
        x, st = s.solve()
        assert st["backward_error"] <= sc.gmres_tolerance
        r = s.calculate_vector_b(x) - s.get_vector_b()
        assert np.linalg.norm(r) <= 10 * sc.gmres_tolerance * np.linalg.norm(s.get_vector_b())


def test_no_illumination_is_an_error(native):
    from itofoggysim_b200 import _native
    sc = S.random_cluster(3, seed=3, p=3)
    with solver.MultiSphereSolver(sc) as s:
        s.set_plane_waves([], [], np.zeros((0, 4)), [], [], np.zeros((0, 3)))
        with pytest.raises(_native.FoggyError):
            s.get_vector_b()
