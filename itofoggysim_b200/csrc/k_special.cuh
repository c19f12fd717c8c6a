// Device special functions shared by the kernels: spherical Bessel/Hankel sequences and
// Wigner small-d tables.  FP64 throughout.
#pragma once

#include "foggy_internal.h"

namespace foggy {

// j_n(x), n = 0..P, single thread.  Forward recurrence where it is stable (x > P), Miller's
// backward recurrence normalised by j_0 or j_1 otherwise (the published methods behind the
// Zhang & Jin SPHJ routine the reference wraps, lib_math_bessel.f90:479-535).
__device__ inline void dev_sph_jn(double x, int P, double* out) {
    double s, c;
    sincos(x, &s, &c);
    double rx = 1.0 / x;
    double j0 = s * rx;
    double j1 = (s * rx - c) * rx;
    out[0] = j0;
    if (P == 0) return;
    if (x > (double)P) {
        out[1] = j1;
        for (int n = 1; n < P; ++n) out[n + 1] = (2.0 * n + 1.0) * rx * out[n] - out[n - 1];
        return;
    }
    int start = P + 16 + (int)x + (int)sqrt(40.0 * (P + x));
    double fnp1 = 0.0, fn = 1e-300;
    for (int n = start; n >= 1; --n) {
        double fnm1 = (2.0 * n + 1.0) * rx * fn - fnp1;
        if (n - 1 <= P) out[n - 1] = fnm1;
        fnp1 = fn;
        fn = fnm1;
        if (fabs(fn) > 1e250) {
            fn *= 1e-250;
            fnp1 *= 1e-250;
            for (int k = n - 1; k <= P; ++k) out[k] *= 1e-250;
        }
    }
    double scale = (fabs(j0) >= fabs(j1)) ? j0 / out[0] : j1 / out[1];
    for (int n = 0; n <= P; ++n) out[n] *= scale;
}

// y_n(x), n = 0..P, forward recurrence (SPHY, lib_math_bessel.f90:593-649).
__device__ inline void dev_sph_yn(double x, int P, double* out) {
    double s, c;
    sincos(x, &s, &c);
    double rx = 1.0 / x;
    out[0] = -c * rx;
    if (P == 0) return;
    out[1] = (-c * rx - s) * rx;
    for (int n = 1; n < P; ++n) out[n + 1] = (2.0 * n + 1.0) * rx * out[n] - out[n - 1];
}

// Quarter table of Wigner small-d: entries d^j_{m' m}(beta) for m' >= |m|, stored at
// dq_index(j, m', m) = j(j+1)(2j+1)/6 + m'(m'+1) + m.
__host__ __device__ __forceinline__ int dq_base(int j) { return j * (j + 1) * (2 * j + 1) / 6; }
__host__ __device__ __forceinline__ int dq_index(int j, int mp, int m) { return dq_base(j) + mp * (mp + 1) + m; }
__host__ __device__ __forceinline__ int dq_size(int pmax) { return dq_base(pmax + 1); }

// d^j_{m' m} for any m', m from the quarter table (symmetries d_{m'm} = (-1)^{m-m'} d_{mm'}
// = d_{-m,-m'}).
__device__ __forceinline__ double dq_get(const double* dq, int j, int mp, int m) {
    int am = m < 0 ? -m : m, amp = mp < 0 ? -mp : mp;
    if (mp >= am) return dq[dq_index(j, mp, m)];
    double sg = ((m - mp) & 1) ? -1.0 : 1.0;
    if (m >= amp) return sg * dq[dq_index(j, m, mp)];
    if (-mp >= am) return sg * dq[dq_index(j, -mp, -m)];
    return dq[dq_index(j, -m, -mp)];
}

__device__ __forceinline__ double ipow_d(double b, int e) {
    double r = 1.0;
    while (e > 0) {
        if (e & 1) r *= b;
        b *= b;
        e >>= 1;
    }
    return r;
}

// One (m', m) column of the quarter table for j = m'..jmax by the upward three-term recurrence
// of the Jacobi polynomials behind d^j_{m'm}.  sqrt_binom[J*(2K+1) + (m+K)] holds
// sqrt((2J)!/((J+m)!(J-m)!)) for K = table width; rs[j*(K+1)+|m|] = sqrt(j^2 - m^2).
__device__ inline void dq_column(double* dq, int mp, int m, int jmax, double cb, double ch, double sh,
                                 const double* sqrt_binom, const double* rs, int K) {
    int J = mp;
    double sg = ((J - m) & 1) ? -1.0 : 1.0;
    double v = sg * sqrt_binom[J * (2 * K + 1) + (m + K)] * ipow_d(ch, J + m) * ipow_d(sh, J - m);
    dq[dq_index(J, mp, m)] = v;
    double prev2 = 0.0, prev1 = v;
    int am = m < 0 ? -m : m;
    for (int j = J + 1; j <= jmax; ++j) {
        double val;
        if (j == 1) {
            val = cb * prev1;
        } else {
            double jj = (double)j;
            double t1 = (cb - (double)(m * mp) / (jj * (jj - 1.0))) * prev1;
            double t2 = rs[(j - 1) * (K + 1) + am] * rs[(j - 1) * (K + 1) + mp] / ((jj - 1.0) * (2.0 * jj - 1.0)) * prev2;
            val = jj * (2.0 * jj - 1.0) / (rs[j * (K + 1) + am] * rs[j * (K + 1) + mp]) * (t1 - t2);
        }
        dq[dq_index(j, mp, m)] = val;
        prev2 = prev1;
        prev1 = val;
    }
}

}  // namespace foggy
