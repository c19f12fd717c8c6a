"""The reference's hcp benchmark scenes (lib_mie_ms_benchmark, FoggySim/src/lib/mie_theory/
lib_mie_multi_sphere.f90:3717-4164) through the device solve and field evaluation, checked
against the oracle: the solution against a dense solve of the oracle operator (1e-5 relative,
the GMRES tolerance is 1e-6) and the scattered field on plot-grid points at 1e-12 of the largest
component for the same coefficients."""
import numpy as np
import pytest

from itofoggysim_b200 import hcp_benchmark, scene as S, solver

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("R", [0.020, 0.0383])
def test_hcp_scene_solve_and_field(native, oracle, R):
    sc = S.hcp_sphere_scene(R)
    P = oracle.Problem(sc)
    with solver.MultiSphereSolver(sc, init_with_single_sphere=True) as s:
        x, st = s.solve()
        assert st["backward_error"] <= 1e-6
        pts, nx, nz = hcp_benchmark.plot_grid(R)
        sel = pts.reshape(-1, 3)[::97]
        E, H = s.get_field(x, sel)
    n = P.n
    A = np.stack([P.matvec(np.eye(n)[i]) for i in range(n)], axis=1)
    xr = np.linalg.solve(A, P.vector_b())
    assert np.linalg.norm(x - xr) <= 1e-5 * np.linalg.norm(xr)
    Eo, Ho = P.field(x, sel)
    assert np.max(np.abs(E - Eo)) <= 1e-12 * np.max(np.abs(Eo))
    assert np.max(np.abs(H - Ho)) <= 1e-12 * np.max(np.abs(Ho))


def test_hcp_benchmark_harness(native, tmp_path):
    hcp_benchmark.main(["--out", str(tmp_path), "--steps", "12", "--last-step", "2", "--operator", "direct"])
    t = np.genfromtxt(str(tmp_path / "hcp_sphere_benchmark_t_matrix.csv"), delimiter=",", skip_header=1)
    assert t.shape == (12, 5) and t[0, 0] == S.hcp_sphere_scene(0.020).n_spheres and np.all(t[:2, 2] > 0)
    for sub in ("real", "realTotal"):
        assert len(list((tmp_path / "t_matrix" / "step_2" / sub).iterdir())) == 30
