"""The single-precision pair tables of the mixed-precision solve stay inside the FP32 range for the
2000-sphere lognormal scenes (CPU, from the FP64 oracle).

The tables hold the coaxial coupling of a sphere pair in the scaled basis x / g_nm,
g_nm = sqrt((n+m)!/(n-m)!).  Their largest entries come from the outgoing radial function h_n at
the largest degree and the smallest separation; spheres do not overlap, so kd >= x_1 + x_2, and
the Wiscombe rule ties each order to its size parameter.  The worst pairs of the distribution are
therefore touching spheres at the radius clips (0.2 and 1.5 um at lambda = 0.55 um).  For each,
the oracle's Xu coefficients on the axis (theta = 0, where only m = mu couples) are scaled to the
device basis and must be finite in float32 with a wide margin, so that products of an entry with
the O(1) scaled coefficients cannot overflow either.
"""
import math

import numpy as np
import pytest

from itofoggysim_b200 import scene as S

LAMBDA = 0.55
R_MIN, R_MAX = 0.2, 1.5   # the lognormal radii's clip of the 2000-sphere scenes


def scaled_axial(oracle, x1, x2):
    """Largest |A|, |B| of the coaxial translation between touching spheres of size parameters x1,
    x2, in the scaled basis of the device (entries for n <= p1, nu <= p2)."""
    p1, p2 = S.wiscombe_n_max(x1), S.wiscombe_n_max(x2)
    A, B = oracle.translation_xu(x1 + x2, 0.0, 0.0, (1, p1), (1, p2), 3)
    g = lambda p: np.array([math.sqrt(math.factorial(n + m) / math.factorial(n - m))
                            for n in range(1, p + 1) for m in range(-n, n + 1)])
    scale = g(p2)[None, :] / g(p1)[:, None]
    return np.max(np.abs(A * scale)), np.max(np.abs(B * scale)), p1, p2


@pytest.mark.parametrize("r1,r2", [(R_MIN, R_MIN), (R_MAX, R_MIN), (R_MAX, R_MAX)])
def test_pair_tables_fit_fp32(oracle, r1, r2):
    k = 2.0 * math.pi / LAMBDA
    a, b, p1, p2 = scaled_axial(oracle, k * r1, k * r2)
    assert np.isfinite(a) and np.isfinite(b)
    big = float(np.finfo(np.float32).max)
    # at least 20 decades of headroom below the largest float32
    assert max(a, b) < big * 1e-20, (p1, p2, a, b)
    assert np.isfinite(np.float32(a)) and np.isfinite(np.float32(b))
