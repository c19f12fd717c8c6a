"""Precision of the 3xTF32 split products that build the single-precision pair tables on the tensor
cores (CPU emulation, against FP64 sums from the oracle's Wigner 3j symbols and Bessel functions).

The table entry of a sphere pair is S(k; a, b) = sum_p G[k, a, b, p] zeta_p with the Gaunt
coefficient G = (2p+1)(a b p; -k k 0)(a b p; 0 0 0) and zeta_p = i^p z_p(kd).  The tensor-core
kernel rounds each operand x to TF32 (10 explicit mantissa bits, round to nearest, ties away) as
hi = tf32(x) and lo = tf32(x - hi), forms hi*hi + hi*lo + lo*hi (each product exact in FP32) and
accumulates in FP32.  Emulated here for the worst pairs of the 2000-sphere lognormal scenes
(touching spheres at the radius clips, 0.2 and 1.5 um at lambda = 0.55 um) and both radial
functions, the table differs from the FP64 sums by less than 5e-7 of its largest entry (6e-8 to
1.6e-7 for these pairs, against 3e-8 to 4.5e-8 for rounding the FP64 sums to FP32); a single TF32
product per term is off by 3e-4 to 5e-4.
"""
import math

import numpy as np
import pytest

from itofoggysim_b200 import scene as S

LAMBDA = 0.55


def tf32(x):
    """Round float32 values to TF32, to nearest with ties away from zero."""
    u = np.asarray(x, dtype=np.float32).view(np.uint32)
    return ((u + np.uint32(0x1000)) & np.uint32(0xFFFFE000)).view(np.float32)


def split(x):
    hi = tf32(np.float32(x))
    lo = tf32(np.float32(x - hi.astype(np.float64)))
    return hi, lo


def pair_block(oracle, ps, pt, kd, z):
    """G[e, p] and zeta_p of the pair block (k = 0..min, a, b = k..M+1), as the kernel lays them out."""
    M2 = max(ps, pt) + 2
    P = 2 * M2 - 2
    jn = oracle.sph_jn(kd, P)
    zeta = jn.astype(complex)
    if z != 1:
        zeta = jn + 1j * oracle.sph_yn(kd, P)
    zeta = zeta * (1j ** np.arange(P + 1))
    rows = []
    for k in range(min(ps, pt) + 1):
        for a in range(k, M2):
            for b in range(k, M2):
                row = np.zeros(P + 1)
                for p in range(abs(a - b), a + b + 1, 2):
                    row[p] = (2 * p + 1) * oracle.wigner_3j(a, b, p, -k, k, 0) * oracle.wigner_3j(a, b, p, 0, 0, 0)
                rows.append(row)
    return np.array(rows), zeta


def emulate_3xtf32(G, zeta):
    """FP32 accumulation, over p, of the three split products of every term."""
    gh, gl = split(G)
    out = []
    for part in (zeta.real, zeta.imag):
        zh, zl = split(part)
        acc = np.zeros(G.shape[0], dtype=np.float32)
        for p in range(G.shape[1]):
            t = (gl[:, p].astype(np.float64) * zh[p] + gh[:, p].astype(np.float64) * zl[p]
                 + gh[:, p].astype(np.float64) * zh[p])
            acc = (acc + t.astype(np.float32)).astype(np.float32)
        out.append(acc.astype(np.float64))
    return out[0] + 1j * out[1]


def one_tf32(G, zeta):
    gh = tf32(np.float32(G)).astype(np.float64)
    return gh @ tf32(np.float32(zeta.real)).astype(np.float64) + 1j * (gh @ tf32(np.float32(zeta.imag)).astype(np.float64))


@pytest.mark.parametrize("z", [1, 3])
@pytest.mark.parametrize("r1,r2", [(0.2, 0.2), (1.5, 0.2), (0.6, 0.6)])
def test_split_products_match_fp64_sums(oracle, r1, r2, z):
    k = 2.0 * math.pi / LAMBDA
    x1, x2 = k * r1, k * r2
    p1, p2 = S.wiscombe_n_max(x1), S.wiscombe_n_max(x2)
    G, zeta = pair_block(oracle, p1, p2, x1 + x2, z)
    ref = G @ zeta
    scale = np.max(np.abs(ref))
    err3 = np.max(np.abs(emulate_3xtf32(G, zeta) - ref)) / scale
    err1 = np.max(np.abs(one_tf32(G, zeta) - ref)) / scale
    assert err3 < 5e-7, (p1, p2, err3)
    assert err1 > 100 * err3, (p1, p2, err1, err3)
