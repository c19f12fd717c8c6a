"""n_max continuation on the device (lib_mie_ms_calculate_scattering_coefficients_ab_nm,
FoggySim/src/lib/mie_theory/lib_mie_multi_sphere.f90:162-371): every path ends with a solve at the
full degree that meets the GMRES tolerance and agrees with a plain solve (1e-6 relative, the
solves stop at a 1e-8 backward error), and leaves the handle at its original degree range."""
import numpy as np
import pytest

from itofoggysim_b200 import scene as S, solver

pytestmark = pytest.mark.gpu


def _scene():
    return S.random_cluster(10, seed=7, p=8, z_coupling=3)


@pytest.mark.parametrize("args,stages", [((4, None, False), [4, 8]), ((2, 2, False), [2, 4, 6, 8]),
                                         ((2, 3, True), None)])
def test_continuation_reaches_plain_solution(native, args, stages):
    sc = _scene()
    with solver.MultiSphereSolver(sc, init_with_single_sphere=True) as s:
        x_ref, st_ref = s.solve()
    with solver.MultiSphereSolver(sc, init_with_single_sphere=True) as s:
        (a, b), st = s.calculate_scattering_coefficients_ab_nm(*args)
        log = s.continuation_log
        assert s.n_range() == (1, 8) and s.n == len(x_ref)
        x = np.stack([a, b], axis=1).reshape(-1)
        assert st["backward_error"] <= sc.gmres_tolerance
        assert np.linalg.norm(x - x_ref) <= 1e-6 * np.linalg.norm(x_ref)
        assert log[-1]["n_max"] == 8 and log[-1]["max_iterations"] == 1000
        if stages is not None:
            assert [e["n_max"] for e in log] == stages
        assert all(e["n_max"] <= 8 for e in log)
        # the handle still solves at the full degree afterwards
        x2, st2 = s.solve()
        assert np.linalg.norm(x2 - x_ref) <= 1e-6 * np.linalg.norm(x_ref)
