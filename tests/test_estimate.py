"""The device-footprint estimate the solve server admits requests by (foggy_estimate_solve_bytes,
host only): the pair-table sizes of the bench scenes, the FP32 tables of a mixed-precision solve,
growth with the Krylov basis, and argument errors."""
import numpy as np
import pytest

from itofoggysim_b200 import _native as N, scene as S, solver


def test_pair_table_sizes_of_the_bench_scenes(native):
    _, tb64 = solver.estimate_solve_bytes(S.small_cluster())
    assert 57e6 < tb64 < 58e6              # 64 spheres of degree 15
    sb, tb = solver.estimate_solve_bytes(S.medium_cluster())
    assert 107e9 < tb < 108e9              # 2000 lognormal spheres, degrees up to 30
    assert 5e9 < sb < 7e9                  # scene, slabs, Krylov basis of GMRES(50), staging


def test_mixed_precision_adds_the_fp32_tables(native):
    sc = S.small_cluster()
    sb0, tb0 = solver.estimate_solve_bytes(sc)
    sb1, tb1 = solver.estimate_solve_bytes(sc, precision=1)
    assert sb1 == sb0 and tb1 == tb0 + tb0 // 2


def test_grows_with_the_krylov_basis(native):
    sc = S.small_cluster()
    sc.gmres_restart = 10
    a, _ = solver.estimate_solve_bytes(sc)
    sc.gmres_restart = 50
    b, _ = solver.estimate_solve_bytes(sc)
    assert b - a >= 40 * 16 * sc.ragged_unknowns()


def test_argument_errors(native):
    sc = S.random_cluster(3, seed=1, p=3)
    sc.param_index = np.array([0, 4, 0], np.int32)
    with pytest.raises(N.FoggyError) as e:
        solver.estimate_solve_bytes(sc)
    assert e.value.code == N.FOGGY_ERR_ARGUMENT
    # degrees run to 45 (the reference's cap); 46 is out of range
    sc = S.random_cluster(3, seed=1, p=3)
    sc.n_range_param = np.array([[1, 46]] * sc.n_param, np.int32)
    sc.n_range = (1, 46)
    with pytest.raises(N.FoggyError) as e:
        solver.estimate_solve_bytes(sc)
    assert e.value.code == N.FOGGY_ERR_ARGUMENT
    sc.n_range_param = np.array([[1, 40]] * sc.n_param, np.int32)
    sc.n_range = (1, 40)
    sb, tb = solver.estimate_solve_bytes(sc)
    assert tb > 0 and sb > 0


def test_mlfmm_adds_its_box_expansions(native):
    """An ML-FMM solve also holds its box expansions and chunk partial sums: more bytes than the
    direct solve, and more again with per-level orders (bounded by the largest order)."""
    sc = S.small_cluster()
    d, _ = solver.estimate_solve_bytes(sc)
    f, _ = solver.estimate_solve_bytes(sc, use_ml_fmm=True)
    f3, _ = solver.estimate_solve_bytes(sc, use_ml_fmm=True, fmm_digits=3.0)
    assert d < f < f3
