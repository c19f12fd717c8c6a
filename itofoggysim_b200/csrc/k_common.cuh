// Small device helpers shared by the operator kernels (index decoding, powers of i, radial
// functions of the coupling).
#pragma once

#include "foggy_kernels.cuh"

namespace foggy {

// i^p c
template <class C>
__device__ __forceinline__ C ipow_mul(int p, C c) {
    switch (p & 3) {
        case 0: return c;
        case 1: return C{-c.y, c.x};
        case 2: return C{-c.x, -c.y};
        default: return C{c.y, -c.x};
    }
}
// t = n^2 - 1 + n + m (n >= 1, -n <= m <= n) -> (n, m)
__device__ __forceinline__ void decode_nm(int t, int& n, int& m) {
    int nn = (int)__fsqrt_rn((float)(t + 1));
    if ((nn + 1) * (nn + 1) <= t + 1) ++nn;
    if (nn * nn > t + 1) --nn;
    n = nn;
    m = t + 1 - nn * nn - nn;
}
// u = 0.. over (n >= 1, 0 <= k <= n) in order -> (n, k)
__device__ __forceinline__ void decode_nk(int u, int& n, int& k) {
    int nn = (int)((-1.0f + __fsqrt_rn(9.0f + 8.0f * (float)u)) * 0.5f);
    if (nn < 1) nn = 1;
    while (nn > 1 && (nn - 1) * (nn + 2) / 2 > u) --nn;
    while (nn * (nn + 3) / 2 <= u) ++nn;
    n = nn;
    k = u - (nn - 1) * (nn + 2) / 2;
}
__device__ __forceinline__ double sgn(int e) { return (e & 1) ? -1.0 : 1.0; }

// zeta_p = i^p z_p(rho) for the radial function selector z (1 j_n, 2 y_n, 3 h1_n, 4 h2_n)
__device__ __forceinline__ cplx zeta_of(int z, int p, const double* jb, const double* yb) {
    cplx zc;
    switch (z) {
        case 1: zc = mk(jb[p], 0.0); break;
        case 2: zc = mk(yb[p], 0.0); break;
        case 3: zc = mk(jb[p], yb[p]); break;
        default: zc = mk(jb[p], -yb[p]); break;
    }
    return ipow_mul(p, zc);
}

}  // namespace foggy
