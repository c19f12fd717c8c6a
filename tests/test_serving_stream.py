"""The serving stream's request generator (scene.serving_request), on the CPU: sphere counts, radii,
wavelengths, volume fractions and right-hand-side counts in their ranges, no overlapping spheres,
and every truncation order within the direct operator's 32."""
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
