"""The algorithmic flop count behind bench.py's roofline (CPU): the closed form over truncation
orders equals an entry-by-entry enumeration of the same definition, the per-translation form
sums to it, and the counts quoted for the two bench scenes hold."""
import os
import sys

import numpy as np
import pytest

from itofoggysim_b200 import scene as S

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


class Orders:
    def __init__(self, p):
        self.p = np.asarray(p, np.int32)

    def p_of_sphere(self):
        return self.p


def enumerate_flops(p):
    """One operator application counted entry by entry: per ordered pair (j <- l) a real d-matrix
    entry times a complex value (4 flops) for every (n, m, m') of the source rotation (degrees
    <= p_l) and of the target rotation (degrees <= p_j), a and b parts; 4 complex MACs (8 flops
    each) per coaxial entry (k, n, nu) with |k| <= n <= p_j, |k| <= nu <= p_l, n, nu >= 1; and the
    T-matrix, one complex multiply (8 flops) per unknown."""
    total = 0
    for j, pj in enumerate(p):
        for l, pl in enumerate(p):
            if j == l:
                continue
            for deg in (pl, pj):
                for n in range(1, deg + 1):
                    for m in range(-n, n + 1):
                        for mp in range(-n, n + 1):
                            total += 2 * 4
            for k in range(-min(pj, pl), min(pj, pl) + 1):
                for n in range(max(1, abs(k)), pj + 1):
                    for nu in range(max(1, abs(k)), pl + 1):
                        total += 4 * 8
        total += 8 * 2 * pj * (pj + 2)
    return total


@pytest.mark.parametrize("p", [[3, 3], [2, 4, 4], [1, 5, 3, 3, 2]])
def test_closed_form_equals_enumeration(p):
    assert bench.algorithmic_flops(Orders(p)) == enumerate_flops(p)


def test_per_translation_form_sums_to_total():
    p = [4, 2, 6, 6, 3]
    per = sum(bench.translation_flops(pj, pl) for j, pj in enumerate(p) for l, pl in enumerate(p) if j != l)
    per += 8 * sum(2 * q * (q + 2) for q in p)
    assert bench.algorithmic_flops(Orders(p)) == per


def test_bench_scene_counts():
    # 64-sphere cluster (p = 15) and the 2000-sphere lognormal cluster, per operator application
    assert bench.algorithmic_flops(S.small_cluster()) == 701184000.0
    assert bench.algorithmic_flops(S.medium_cluster()) == pytest.approx(1.0793e12, rel=1e-4)
