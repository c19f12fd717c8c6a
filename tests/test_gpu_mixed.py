"""Mixed-precision solves (foggy_params.precision = 1): Arnoldi steps with the FP32 operator, true
residuals with the FP64 operator at the start and at every restart.  The solve must reach the same
FP64 backward error as the FP64 solve, and its solution and extinction cross-section must agree
with the FP64 ones to the level that tolerance allows (1e-6 relative on the coefficients for a
1e-8 residual, 1e-7 on C_ext)."""
import numpy as np
import pytest

from itofoggysim_b200 import _native as N, scene as S, solver

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["small_cluster", "polydisperse"])
@pytest.mark.parametrize("tables", [0, 1])
def test_mixed_solve_matches_fp64(native, case, tables):
    sc = S.small_cluster() if case == "small_cluster" else S.random_cluster(40, seed=6, p=None, z_coupling=3)
    with solver.MultiSphereSolver(sc, pair_tables=tables) as s:
        x64, st64 = s.solve()
        c64 = s.cross_sections(x64)
        b = s.get_vector_b()
        r64 = s.calculate_vector_b(x64) - b
    with solver.MultiSphereSolver(sc, pair_tables=tables, precision=1) as s:
        x32, st32 = s.solve()
        c32 = s.cross_sections(x32)
        r32 = s.calculate_vector_b(x32) - b
    # the device's backward error (FP64 operator, scaled basis x / g_nm) meets the tolerance; in the
    # reference layout the residual is of the size the FP64 solve leaves there
    assert st32["backward_error"] <= sc.gmres_tolerance
    assert np.linalg.norm(r32) <= 10 * np.linalg.norm(r64) + 1e-14 * np.linalg.norm(b)
    assert np.linalg.norm(x32 - x64) <= 1e-6 * np.linalg.norm(x64)
    assert abs(c32[1] - c64[1]) <= 1e-7 * abs(c64[1])
    assert st32["restarts"] >= 1


@pytest.mark.parametrize("tables", [0, -1])
def test_mixed_mlfmm_solve_matches_fp64(native, tables):
    """The ML-FMM passes in FP32 in the Arnoldi steps (consistent convention, a scene whose boxes
    are small against the wavelength): FP64 backward error met, solution within 1e-6 and C_ext within
    1e-7 of the FP64 ML-FMM solve, with the cached translation blocks and without."""
    rng = np.random.default_rng(7)
    sc = S.make_scene(rng.uniform(0.1, 0.3, 40), 10.0, 5, lambda_0=6.0, n_max=8, z_coupling=3,
                      reference_row_rule=False, tree_l_max=3, gmres_tolerance=1e-8)
    with solver.MultiSphereSolver(sc, use_ml_fmm=True, fmm_convention=1, pair_tables=tables) as s:
        x64, st64 = s.solve()
        c64 = s.cross_sections(x64)
    with solver.MultiSphereSolver(sc, use_ml_fmm=True, fmm_convention=1, pair_tables=tables, precision=1) as s:
        x32, st32 = s.solve()
        c32 = s.cross_sections(x32)
    assert st64["status"] == 0 and st32["status"] == 0
    assert st32["backward_error"] <= sc.gmres_tolerance
    assert np.linalg.norm(x32 - x64) <= 1e-6 * np.linalg.norm(x64)
    assert abs(c32[1] - c64[1]) <= 1e-7 * abs(c64[1])