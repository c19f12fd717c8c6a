"""The oracle's octree lists and ML-FMM (test infrastructure), on the CPU.

Pins: the neighbour lists, parent and children numbering of the reference's own tree tests
(libtree/src/lib/lib_tree_helper_functions.f90:2277-2356, 2399-2579, via tests/golden); the
interaction list follows from them (children of the parent's neighbourhood minus the own
neighbourhood, lib_tree.f90:994-1143).  The oracle ML-FMM in its consistent convention must
tend to the direct operator as the expansion order grows, which checks the tree lists and the
pass structure (aggregation, M2M, M2L, L2L, box-to-sphere, near field) end to end.
"""
import math

import numpy as np

from itofoggysim_b200 import scene as S

CENTRES = np.random.default_rng(0).uniform(0.0, 10.0, (40, 3))


def test_neighbours_match_reference(oracle, golden):
    for case in golden["tree_neighbours"]:
        got = oracle.tree_domain(CENTRES, 3, case["l"], case["n"], 3)
        assert sorted(got.tolist()) == sorted(case["neighbours"])


def test_interaction_list_from_reference_rules(oracle, golden):
    # level-2 box 35: its parent (35 >> 3 = 4, the reference's parent rule, golden 6 -> 0) has all
    # eight level-1 boxes as neighbourhood, whose children (8 c .. 8 c + 7, golden 1 -> 8..15) are all
    # 64 level-2 boxes; minus box 35 and its 26 neighbours
    assert golden["tree_parent"]["parent"] == golden["tree_parent"]["n"] >> 3
    assert golden["tree_children"]["children"] == [(golden["tree_children"]["n"] << 3) | c for c in range(8)]
    nb = next(c for c in golden["tree_neighbours"] if c["l"] == 2 and c["n"] == 35)["neighbours"]
    expect = sorted(set(range(64)) - set(nb) - {35})
    assert oracle.tree_domain(CENTRES, 3, 2, 35, 4).tolist() == expect
    # an interior box at level 3 has the full 6^3 - 3^3 = 189 boxes
    c = (3, 3, 3)
    n = 0
    for b in range(3):
        for d in range(3):
            n |= ((c[d] >> b) & 1) << (3 * b + (2 - d))
    assert len(oracle.tree_domain(CENTRES, 3, 3, n, 4)) == 189


def test_e1_partitions_spheres_and_e2_contains_e1(oracle):
    u = [oracle.universal_index(c, 2) for c in oracle.scale_points(CENTRES)]
    seen = []
    for n in sorted(set(u)):
        e1 = oracle.tree_domain(CENTRES, 3, 2, n, 1).tolist()
        e2 = set(oracle.tree_domain(CENTRES, 3, 2, n, 2).tolist())
        assert sorted(e1) == sorted(i for i, v in enumerate(u) if v == n)
        assert set(e1) <= e2
        seen += e1
    assert sorted(seen) == list(range(len(CENTRES)))


def _g(sc):
    g = [math.sqrt(math.factorial(n + m) / math.factorial(n - m))
         for n in range(1, sc.n_range[1] + 1) for m in range(-n, n + 1)]
    return np.tile(np.concatenate([g, g]), sc.n_spheres)


def long_wave_scene(p, z=3, n=20):
    """20 small spheres in an 8 um cube at lambda = 6 um: boxes a fraction of a wavelength."""
    rng = np.random.default_rng(7)
    radii = rng.uniform(0.1, 0.3, n)
    return S.make_scene(radii, 8.0, 5, lambda_0=6.0, n_max=p, z_coupling=z, reference_row_rule=False,
                        tree_l_max=3)


def test_consistent_fmm_tends_to_direct(oracle):
    errs = []
    for p in (4, 8):
        sc = long_wave_scene(p)
        P = oracle.Problem(sc)
        rng = np.random.default_rng(1)
        x = (rng.standard_normal(sc.vector_length()) + 1j * rng.standard_normal(sc.vector_length())) * _g(sc)
        yd = P.matvec(x)
        yf = P.fmm_matvec(x, l_max=3, convention=1)
        g = _g(sc)
        errs.append(np.max(np.abs((yf - yd) / g)) / np.max(np.abs(yd / g)))
    assert errs[1] < 2e-3
    assert errs[1] < errs[0] / 10


def test_per_level_orders_closer_to_direct(oracle):
    """Per-level expansion orders (digits > 0: the excess-bandwidth order of each level's box diagonal,
    never below the global order; not in the reference) bring the consistent expansion closer to the
    direct operator than the global order alone; digits = 0 is the global order itself."""
    sc = long_wave_scene(4)
    P = oracle.Problem(sc)
    rng = np.random.default_rng(2)
    x = (rng.standard_normal(sc.vector_length()) + 1j * rng.standard_normal(sc.vector_length())) * _g(sc)
    yd = P.matvec(x)
    y0 = P.fmm_matvec(x, l_max=3, convention=1)
    assert np.array_equal(P.fmm_matvec(x, l_max=3, convention=1, digits=0.0), y0)
    y3 = P.fmm_matvec(x, l_max=3, convention=1, digits=3.0)
    g = _g(sc)
    err = lambda y: np.max(np.abs((y - yd) / g)) / np.max(np.abs(yd / g))
    assert err(y3) < err(y0)
