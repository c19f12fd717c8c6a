"""bench.py's workload definitions on the CPU.  The algorithmic flop count behind the roofline: the
closed form over truncation orders equals an entry-by-entry enumeration of the same definition,
the per-translation form sums to it, and the counts quoted for the two bench scenes hold.  The
128 right-hand sides of the several-right-hand-side workload: Fibonacci directions x TM/TE."""
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


def test_fibonacci_right_hand_sides():
    # 64 directions z_i = 1 - (2i+1)/64, phi_i = i pi (3 - sqrt 5) (mod 2 pi), each TM then TE
    w = bench.fibonacci_waves(64)
    i = np.arange(64)
    assert len(w["wave_theta"]) == 128
    assert np.allclose(np.cos(w["wave_theta"][::2]), 1.0 - (2.0 * i + 1.0) / 64.0, atol=1e-15)
    assert np.allclose(w["wave_phi"][::2], np.mod(i * np.pi * (3.0 - np.sqrt(5.0)), 2.0 * np.pi), atol=1e-12)
    assert np.array_equal(w["wave_theta"][::2], w["wave_theta"][1::2])
    assert np.all(w["jones"][::2] == [1.0, 0.0, 0.0, 0.0]) and np.all(w["jones"][1::2] == [0.0, 0.0, 1.0, 0.0])
    d = np.stack([np.sin(w["wave_theta"][::2]) * np.cos(w["wave_phi"][::2]),
                  np.sin(w["wave_theta"][::2]) * np.sin(w["wave_phi"][::2]), np.cos(w["wave_theta"][::2])], 1)
    # distinct directions, spread over the sphere (mean direction near zero)
    assert np.min(np.linalg.norm(d[:, None] - d[None], axis=-1) + 10 * np.eye(64)) > 0.2
    assert np.linalg.norm(d.mean(0)) < 0.05


def test_block_workload_scene():
    """The block workload: the 20,000-sphere scene's shape (lognormal radii at 20,000 spheres per 90 um cube)
    at a smaller sphere count, 128 right-hand sides, GMRES(30) to 1e-6."""
    sc = bench.block_scene(500)
    assert sc.n_spheres == 500 and sc.n_waves == 128
    assert sc.gmres_tolerance == 1e-6 and sc.gmres_restart == 30
    edge = 90.0 * (500 / 20000.0) ** (1.0 / 3.0)
    assert np.all(sc.centres >= 0.0) and np.all(sc.centres < edge)
    p = sc.p_of_sphere()
    assert p.max() <= 30 and 15 <= np.median(p) <= 19


def test_cached_operator_size_and_scale():
    """The cached CPU operator keeps two P_j x P_l complex blocks per ordered pair; its work goes with
    sum_{j != l} P_j P_l."""
    a, b = Orders([3, 3, 5]), Orders([3, 5, 5, 5])
    P = lambda o: [int(v) * (int(v) + 2) for v in o.p]
    def pairs(o):
        q = P(o)
        return sum(q[i] * q[j] for i in range(len(q)) for j in range(len(q)) if i != j)
    assert bench.cached_bytes(a) == 32 * pairs(a)
    assert abs(bench.cached_scale(a, b) - pairs(b) / pairs(a)) < 1e-12
    # the 64-sphere cluster's cache: 4032 pairs x 2 x 255^2 x 16 bytes
    assert bench.cached_bytes(S.small_cluster()) == 4032 * 2 * 255 ** 2 * 16


def test_long_wave_scene():
    """The ML-FMM comparison scene: spheres of radius 0.1-0.3 um at lambda = 6 um, 0.04 per um^3,
    global order 8."""
    sc = bench.long_wave_scene(500)
    assert sc.n_spheres == 500 and sc.lambda_0 == 6.0
    assert np.all(sc.p_of_sphere() == 8)
    edge = (500 / 0.04) ** (1.0 / 3.0)
    assert np.all(sc.centres >= 0.0) and np.all(sc.centres < edge)
    assert np.all((sc.radius >= 0.1) & (sc.radius <= 0.3))
