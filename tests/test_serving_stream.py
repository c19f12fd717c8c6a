"""The synthetic workloads on the CPU.  The serving stream's request generator
(scene.serving_request): sphere counts, radii, wavelengths, volume fractions and right-hand-side
counts in their ranges, no overlapping spheres, and every truncation order within the direct
operator's 32.  The two bench scenes: sizes and truncation-order statistics."""
import math

import numpy as np

from itofoggysim_b200 import scene as S


def test_requests_stay_in_their_ranges():
    rng = np.random.default_rng(42)
    counts = []
    for _ in range(60):
        sc = S.serving_request(rng)
        n = sc.n_spheres
        counts.append(n)
        assert 50 <= n <= 500
        r = sc.radius[sc.param_index]
        assert r.min() >= 0.2 and r.max() <= 1.2
        assert 0.45 <= sc.lambda_0 <= 0.65
        assert 1 <= sc.n_waves <= 16
        assert sc.p_of_sphere().max() <= 32
        edge = np.ptp(sc.centres, axis=0).max() + 2 * r.max()
        vf = np.sum(4.0 / 3.0 * math.pi * r ** 3) / edge ** 3
        assert 0.005 <= vf <= 0.06
        d = np.linalg.norm(sc.centres[:, None] - sc.centres[None], axis=-1) + 1e9 * np.eye(n)
        assert np.all(d >= r[:, None] + r[None])
    # log-uniform counts: as many requests below the geometric middle of [50, 500] as above it
    below = np.mean(np.array(counts) < math.sqrt(50 * 500))
    assert 0.3 < below < 0.7


def test_bench_scenes():
    # 64 water spheres of r = 0.5 um in a 10 um cube, p = 15 each: 32,640 unknowns
    sc = S.small_cluster()
    assert sc.n_spheres == 64 and np.all(sc.p_of_sphere() == 15) and sc.vector_length() == 32640
    # 2000 lognormal spheres (median 0.6 um, sigma_ln 0.3, clipped to 0.2-1.5 um) in a 40 um cube:
    # per-sphere Wiscombe orders with median 17, 95th percentile 23 and maximum 30
    sc = S.medium_cluster()
    p = sc.p_of_sphere()
    r = sc.radius[sc.param_index]
    assert sc.n_spheres == 2000 and r.min() >= 0.2 and r.max() <= 1.5
    assert np.median(p) == 17 and np.percentile(p, 95) == 23 and p.max() == 30
    assert np.all(sc.centres >= 0.0) and np.all(sc.centres <= 40.0)
    assert sc.ragged_unknowns() == 1365282
