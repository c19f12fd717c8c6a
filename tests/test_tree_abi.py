"""libtree box arithmetic through the C ABI (host functions, no GPU): parent, children, centre of
box and neighbours, pinned by the reference's own tree tests (libtree/src/lib/lib_tree_helper_functions.f90:
parent and children :2277-2356, centre of box :2358-2397, neighbours :2399-2579, interleave :3003-3040,
de-interleave :3088-3130) and checked against the oracle's neighbour lists."""
import numpy as np
import pytest

from itofoggysim_b200 import _native as N, solver


def test_parent_children_golden(native, golden):
    g = golden["tree_parent"]
    assert solver.tree_parent(g["n"], g["l"]) == g["parent"]
    g = golden["tree_children"]
    assert solver.tree_children(g["n"], 1).tolist() == g["children"]


def test_neighbours_golden(native, golden):
    for case in golden["tree_neighbours"]:
        assert solver.tree_neighbours(case["n"], case["l"]).tolist() == sorted(case["neighbours"])


def test_centre_of_box_golden(native):
    # lib_tree_helper_functions.f90:2358-2397, compared for equality as the reference does
    assert solver.tree_centre_of_box(1, 1).tolist() == [0.25, 0.25, 0.75]
    # de-interleave 2^0 + 2^5 -> coordinates (2, 0, 1) (:3088-3130)
    assert solver.tree_centre_of_box(2 ** 0 + 2 ** 5, 2).tolist() == [2.5 / 4, 0.5 / 4, 1.5 / 4]
    # interleave (2^0 + 2^5, 2^2 + 2^4, 2^1 + 2^6) -> 2^2 + 2^3 + 2^7 + 2^13 + 2^17 + 2^18 (:3003-3040)
    n = 2 ** 2 + 2 ** 3 + 2 ** 7 + 2 ** 13 + 2 ** 17 + 2 ** 18
    c = np.array([2 ** 0 + 2 ** 5, 2 ** 2 + 2 ** 4, 2 ** 1 + 2 ** 6]) + 0.5
    assert solver.tree_centre_of_box(n, 7).tolist() == (c / 2 ** 7).tolist()


def test_neighbours_match_oracle(native, oracle):
    centres = np.random.default_rng(0).uniform(0.0, 10.0, (40, 3))
    for l in (1, 2, 3):
        for n in range(0, 8 ** l, max(1, 8 ** l // 64)):
            want = sorted(oracle.tree_domain(centres, 3, l, n, 3).tolist())
            assert solver.tree_neighbours(n, l).tolist() == want, (l, n)


def test_parent_of_children_and_steps(native):
    rng = np.random.default_rng(5)
    for l in (1, 5, 12, 20):
        for n in rng.integers(0, 8 ** l, 20):
            assert all(solver.tree_parent(c, l + 1) == n for c in solver.tree_children(n, l))
            assert solver.tree_parent(n, l, l) == 0
            if l > 2:
                assert solver.tree_parent(n, l, 2) == int(n) >> 6


def test_deepest_level(native):
    n = 2 ** 63 - 1   # the last level-21 box
    c = solver.tree_centre_of_box(n, 21)
    assert np.all(c == (2 ** 21 - 0.5) / 2 ** 21)
    assert len(solver.tree_neighbours(n, 21)) == 7
    assert solver.tree_parent(n, 21) == 2 ** 60 - 1


@pytest.mark.parametrize("call", [
    lambda: solver.tree_parent(0, 22),
    lambda: solver.tree_parent(-1, 3),
    lambda: solver.tree_parent(64, 2),
    lambda: solver.tree_parent(5, 2, 0),
    lambda: solver.tree_parent(5, 2, 3),
    lambda: solver.tree_children(0, 21),
    lambda: solver.tree_centre_of_box(8, 1),
    lambda: solver.tree_neighbours(512, 3),
])
def test_argument_errors(native, call):
    with pytest.raises(N.FoggyError) as e:
        call()
    assert e.value.code == N.FOGGY_ERR_ARGUMENT
