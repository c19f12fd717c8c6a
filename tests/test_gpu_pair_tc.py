"""Single-precision pair tables as tensor-core products (tcgen05.mma kind::tf32, 3xTF32).

A handle in mixed precision (precision = 1) keeps its FP32 pair tables, the scalar coaxial
coefficients S(k; a, b) of every sphere pair, as the product of the Gaunt coefficients and the
pairs' i^p z_p(kd) on the tensor cores, each operand split into a TF32 high and low part
(k_pair_tables.cu).  The FP32 operator that reads those tables must agree with

  * the FP64 operator of the same handle (FP64 tables summed in FP64, pinned to the oracle at 1e-12
    by test_gpu_parity.py and test_gpu_high_order.py): 1e-5, the tolerance of every FP32 operator
    test (test_gpu_block.py);
  * the FP32 operator without tables, which sums S per pair on every application: 1e-5;

and two handles must build bit-identical tables (the same operator output bit for bit).

Scenes: orders 3..15 with 150 spheres (several tiles of 64 pairs per group, partial last tiles),
orders 17..30 (the upper buckets of the benchmark's lognormal scene), orders 34 and 45 (K > 72:
tiles of 16 pairs), z = j_n and h_n.

Error metric: vectors divided by g_nm (the basis the device works in), max |x - ref| / max |ref|.
"""
import math

import numpy as np
import pytest

from itofoggysim_b200 import scene as S, solver

pytestmark = pytest.mark.gpu

TOL_FP32 = 1e-5


def _g_layout(sc):
    g = np.array([math.sqrt(math.factorial(n + m) / math.factorial(n - m))
                  for n in range(1, sc.n_range[1] + 1) for m in range(-n, n + 1)])
    return np.tile(np.concatenate([g, g]), sc.n_spheres)


def _err(x, ref, g):
    a, r = x / g, ref / g
    return np.max(np.abs(a - r)) / max(np.max(np.abs(r)), 1e-300)


def _vectors(sc, nv, seed):
    rng = np.random.default_rng(seed)
    g = _g_layout(sc)
    n = sc.vector_length()
    X = (rng.standard_normal((nv, n)) + 1j * rng.standard_normal((nv, n))) * g
    C = (sc.n_range[1] + 1) ** 2 - 1
    p = sc.p_of_sphere()
    Xv = X.reshape(nv, sc.n_spheres, 2, C)
    for j in range(sc.n_spheres):
        Xv[:, j, :, p[j] * (p[j] + 2):] = 0
    return X


SCENES = {
    "many_pairs": lambda z: S.random_cluster(150, seed=51, p=None, z_coupling=z, reference_row_rule=False),
    "orders_17_30": lambda z: S.random_cluster(6, seed=41, radii=np.array([0.6, 0.7, 0.95, 1.15, 1.3, 1.5]),
                                               box=8.0, z_coupling=z, reference_row_rule=False),
    "orders_34_45": lambda z: S.random_cluster(3, seed=43, radii=np.array([1.8, 2.6, 0.5]), box=10.0,
                                               z_coupling=z, reference_row_rule=False),
}


@pytest.mark.parametrize("z", [1, 3])
@pytest.mark.parametrize("case", sorted(SCENES))
def test_tensor_core_tables_operator(native, case, z):
    sc = SCENES[case](z)
    g = _g_layout(sc)
    X = _vectors(sc, 3, 17)
    with solver.MultiSphereSolver(sc, precision=1, pair_tables=1) as s:
        Y64 = np.stack([s.calculate_vector_b(x) for x in X])
        Ytc = s.calculate_vector_b_block(X, precision=1)
    with solver.MultiSphereSolver(sc, precision=1, pair_tables=1) as s:
        Ytc2 = s.calculate_vector_b_block(X, precision=1)
    with solver.MultiSphereSolver(sc, precision=1, pair_tables=-1) as s:
        Ysum = s.calculate_vector_b_block(X, precision=1)
    assert np.array_equal(Ytc, Ytc2), "tensor-core tables differ between two builds"
    for v in range(len(X)):
        e64, esum = _err(Ytc[v], Y64[v], g), _err(Ytc[v], Ysum[v], g)
        assert np.all(np.isfinite(Ytc[v]))
        assert e64 < TOL_FP32, (v, e64)
        assert esum < TOL_FP32, (v, esum)


def test_tensor_core_tables_mixed_solve(native):
    """A mixed-precision solve on the tensor-core tables meets the FP64 tolerance (its restarts
    refine with the FP64 operator) and agrees with the FP64 solve to 1e-6."""
    sc = S.random_cluster(40, seed=52, p=None, z_coupling=3, reference_row_rule=False)
    sc.gmres_tolerance = 1e-10
    g = _g_layout(sc)
    with solver.MultiSphereSolver(sc, pair_tables=1) as s:
        x64, st64 = s.solve()
    with solver.MultiSphereSolver(sc, pair_tables=1, precision=1) as s:
        x32, st32 = s.solve()
    assert st64["status"] == 0 and st32["status"] == 0
    assert st32["backward_error"] <= 1e-10
    assert np.linalg.norm((x32 - x64) / g) / np.linalg.norm(x64 / g) < 1e-6
