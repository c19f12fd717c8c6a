// FP64 CPU ORACLE -- test infrastructure only.
//
// This file restates, in C++, the reference algorithms of ItoFoggySim's multi-sphere Mie
// solve so that the CUDA implementation can be checked against them.  It is linked only by
// the tests, by __graft_entry__.smoke() and by the CPU-baseline leg of bench.py.  Nothing in
// the product library calls into it.
//
// Every function cites the reference file:line it follows (paths relative to the reference
// project root).  The Wigner-3j symbols come from the reference's own C library wigxjpf 1.10
// (wigxjpf_1_10/src), compiled from its sources into oracle/_ref/ by oracle/Makefile.
//
// Conventions (identical to the reference):
//   * complex numbers are two interleaved doubles (Fortran complex(8));
//   * a per-sphere coefficient block is [a_nm | b_nm], each ordered n = n1..n2, m = -n..n
//     (lib_mie_ms_solver_interface_helper_functions.f90:49-163,
//      lib_math_type_operator.f90:2600-2730);
//   * associated Legendre functions carry no Condon-Shortley phase (LPMNS convention,
//     lib_math_legendre.f90:68-313).

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>
#include <map>
#include <array>
#include <omp.h>

extern "C" {
void wig_table_init(int max_two_j, int wigner_type);
void wig_thread_temp_init(int max_two_j);
void wig_temp_free(void);
double wig3jj(int two_j1, int two_j2, int two_j3, int two_m1, int two_m2, int two_m3);
}

// wigxjpf keeps one scratch array per thread (wig_thread_temp_init allocates a new one each call).
// Grow the calling thread's array when it is smaller than asked, never shrink it: the main thread
// also runs in the OpenMP regions below, and a smaller array left there would make a later 3j call
// of higher degree on that thread fail.
static void ensure_wig_temp(int max_two_j) {
    static thread_local int have = -1;
    if (have >= max_two_j) return;
    if (have >= 0) wig_temp_free();
    wig_thread_temp_init(max_two_j);
    have = max_two_j;
}

typedef std::complex<double> cd;
static const double PI = 3.14159265358979323846264338327950288;

namespace {

// ------------------------------------------------------------------------------------------
// factorial ratios  (libmath/src/math/lib_math_factorial.f90:102-290; the cache bound is
// never assigned there, so the uncached product form is what runs)
// ------------------------------------------------------------------------------------------
double fact(int n) {
    double r = 1.0;
    for (int i = 2; i <= n; ++i) r *= i;
    return r;
}
// (n-m)!/(n+m)!
double nmm_over_npm(int n, int m) {
    if (m >= 0) {
        if (n == m) return 1.0 / fact(n + m);
        double r = 1.0;
        for (int i = n - m + 1; i <= n + m; ++i) r *= i;
        return 1.0 / r;
    }
    // (n+|m|)!/(n-|m|)!
    int a = -m;
    double r = 1.0;
    for (int i = n - a + 1; i <= n + a; ++i) r *= i;
    return r;
}
// (n+m)!/(n-m)!
double npm_over_nmm(int n, int m) { return nmm_over_npm(n, -m); }

// ------------------------------------------------------------------------------------------
// spherical Bessel functions (lib_math_bessel.f90:479-789 wraps Zhang & Jin SPHJ/SPHY, which
// are not vendored; restated with the published methods: Miller backward recurrence for j_n
// normalised by j_0 or j_1, forward recurrence for y_n)
// ------------------------------------------------------------------------------------------
void sph_jn(double x, int nmax, double* out) {
    if (x == 0.0) {
        for (int n = 0; n <= nmax; ++n) out[n] = (n == 0) ? 1.0 : 0.0;
        return;
    }
    double j0 = std::sin(x) / x;
    double j1 = std::sin(x) / (x * x) - std::cos(x) / x;
    if (nmax == 0) { out[0] = j0; return; }
    int start = nmax + 16 + (int)(x) + (int)(std::sqrt(40.0 * (nmax + x)));
    std::vector<double> f(start + 2, 0.0);
    f[start + 1] = 0.0;
    f[start] = 1e-300;
    for (int n = start; n >= 1; --n) {
        f[n - 1] = (2.0 * n + 1.0) / x * f[n] - f[n + 1];
        if (std::fabs(f[n - 1]) > 1e250) {
            for (int k = n - 1; k <= start + 1; ++k) f[k] *= 1e-250;
        }
    }
    double scale = (std::fabs(j0) >= std::fabs(j1)) ? j0 / f[0] : j1 / f[1];
    for (int n = 0; n <= nmax; ++n) out[n] = f[n] * scale;
}

void sph_yn(double x, int nmax, double* out) {
    double y0 = -std::cos(x) / x;
    out[0] = y0;
    if (nmax == 0) return;
    double y1 = -std::cos(x) / (x * x) - std::sin(x) / x;
    out[1] = y1;
    for (int n = 1; n < nmax; ++n) out[n + 1] = (2.0 * n + 1.0) / x * out[n] - out[n - 1];
}

// z_n for the translation selector (lib_math_vector_spherical_harmonics.f90:1420-1448):
// 1 j_n, 2 y_n, 3 h^(1)_n = j_n + i y_n, 4 h^(2)_n = j_n - i y_n
void sph_z(int z, double x, int nmax, cd* out) {
    std::vector<double> j(nmax + 1), y(nmax + 1);
    sph_jn(x, nmax, j.data());
    if (z != 1) sph_yn(x, nmax, y.data());
    for (int n = 0; n <= nmax; ++n) {
        switch (z) {
            case 1: out[n] = cd(j[n], 0.0); break;
            case 2: out[n] = cd(y[n], 0.0); break;
            case 3: out[n] = cd(j[n], y[n]); break;
            default: out[n] = cd(j[n], -y[n]); break;
        }
    }
}

// ------------------------------------------------------------------------------------------
// associated Legendre functions without Condon-Shortley phase, including negative orders
// (lib_math_legendre.f90:128-313; LPMNS recurrence for m >= 0, P_n^{-m} = (-1)^m
// (n-m)!/(n+m)! P_n^m).  Table P[n*(n+1)+m] for n = 0..nmax, m = -n..n.
// ------------------------------------------------------------------------------------------
void legendre_table(double x, int nmax, double* P) {
    double s = std::sqrt(std::fabs(1.0 - x * x));
    for (int m = 0; m <= nmax; ++m) {
        double pmm = 1.0;
        for (int k = 1; k <= m; ++k) pmm = (2.0 * k - 1.0) * s * pmm;
        double pk2 = pmm, pk1 = 0.0;
        P[m * (m + 1) + m] = pmm;
        if (m + 1 <= nmax) {
            pk1 = (2.0 * m + 1.0) * x * pmm;
            P[(m + 1) * (m + 2) + m] = pk1;
        }
        for (int k = m + 2; k <= nmax; ++k) {
            double pk = ((2.0 * k - 1.0) * x * pk1 - (k + m - 1.0) * pk2) / (k - m);
            P[k * (k + 1) + m] = pk;
            pk2 = pk1;
            pk1 = pk;
        }
        if (m > 0) {
            for (int k = m; k <= nmax; ++k) {
                double f = nmm_over_npm(k, m);
                if (m & 1) f = -f;
                P[k * (k + 1) - m] = f * P[k * (k + 1) + m];
            }
        }
    }
}

// pi_nm = m P_n^m(cos t)/sin t and tau_nm = dP_n^m(cos t)/dt without Condon-Shortley phase
// (lib_math_legendre.f90:834-982, "theta_wa"; the reference evaluates generated closed forms
// and removes the phase for odd |m|).  With cs_phase != 0 the phase is kept, which is the
// form of the golden values at lib_math_legendre.f90:2099-2210.  The poles use the
// reference's special values (lib_math_legendre.f90:854-920).  Table index n*(n+1)+m.
void pi_tau_table(double theta, int nmax, int cs_phase, double* pi, double* tau) {
    int sz = (nmax + 1) * (nmax + 1);
    std::fill(pi, pi + sz, 0.0);
    std::fill(tau, tau + sz, 0.0);
    double x = std::cos(theta);
    if (x == 1.0 || x == -1.0) {
        // values with Condon-Shortley phase, as in the reference before its phase removal
        for (int n = 1; n <= nmax; ++n) {
            pi[n * (n + 1) - 1] = -0.5;
            pi[n * (n + 1) + 1] = -(double)(n * (n + 1) / 2);
        }
        if (x == -1.0)
            for (int n = 2; n <= nmax; n += 2) {
                pi[n * (n + 1) - 1] = -pi[n * (n + 1) - 1];
                pi[n * (n + 1) + 1] = -pi[n * (n + 1) + 1];
            }
        for (int n = 1; n <= nmax; ++n) {
            tau[n * (n + 1) - 1] = 0.5;
            tau[n * (n + 1) + 1] = -(double)(n * (n + 1) / 2);
        }
        if (x == -1.0)
            for (int n = 1; n <= nmax; n += 2) {   // the reference copies -pi here
                tau[n * (n + 1) - 1] = -pi[n * (n + 1) - 1];
                tau[n * (n + 1) + 1] = -pi[n * (n + 1) + 1];
            }
        if (!cs_phase)
            for (int n = 1; n <= nmax; ++n) {
                pi[n * (n + 1) - 1] = -pi[n * (n + 1) - 1];
                pi[n * (n + 1) + 1] = -pi[n * (n + 1) + 1];
                tau[n * (n + 1) - 1] = -tau[n * (n + 1) - 1];
                tau[n * (n + 1) + 1] = -tau[n * (n + 1) + 1];
            }
        return;
    }
    double s = std::sin(theta);
    // no-phase values: Q_n^m = P_n^m / sin t for m >= 1 by the LPMNS recurrence
    std::vector<double> Q((nmax + 2) * (nmax + 2), 0.0);
    std::vector<double> P((nmax + 2) * (nmax + 2), 0.0);
    legendre_table(x, nmax + 1, P.data());
    for (int m = 1; m <= nmax; ++m) {
        double qmm = 1.0;
        for (int k = 1; k <= m; ++k) qmm *= (2.0 * k - 1.0);
        for (int k = 1; k < m; ++k) qmm *= s;
        double q2 = qmm, q1 = 0.0;
        Q[m * (m + 1) + m] = qmm;
        if (m + 1 <= nmax) {
            q1 = (2.0 * m + 1.0) * x * qmm;
            Q[(m + 1) * (m + 2) + m] = q1;
        }
        for (int k = m + 2; k <= nmax; ++k) {
            double qk = ((2.0 * k - 1.0) * x * q1 - (k + m - 1.0) * q2) / (k - m);
            Q[k * (k + 1) + m] = qk;
            q2 = q1;
            q1 = qk;
        }
    }
    for (int n = 1; n <= nmax; ++n) {
        // m = 0: pi = 0, tau = dP_n/dt = -P_n^1 (no phase)
        tau[n * (n + 1)] = -P[n * (n + 1) + 1];
        for (int m = 1; m <= n; ++m) {
            double qn = Q[n * (n + 1) + m];
            double qn1 = (n - 1 >= m) ? Q[(n - 1) * n + m] : 0.0;
            double pv = m * qn;
            double tv = n * x * qn - (n + m) * qn1;
            double f = nmm_over_npm(n, m);
            if (m & 1) f = -f;
            pi[n * (n + 1) + m] = pv;
            tau[n * (n + 1) + m] = tv;
            pi[n * (n + 1) - m] = -f * pv;   // (-m) P_n^{-m} / sin t
            tau[n * (n + 1) - m] = f * tv;
        }
    }
    if (cs_phase)
        for (int n = 1; n <= nmax; ++n)
            for (int m = -n; m <= n; ++m)
                if (std::abs(m) & 1) {
                    pi[n * (n + 1) + m] = -pi[n * (n + 1) + m];
                    tau[n * (n + 1) + m] = -tau[n * (n + 1) + m];
                }
}

// ------------------------------------------------------------------------------------------
// Wigner 3j through the reference's wigxjpf (libmath/src/math/lib_math_wigner.f90:45-72)
// ------------------------------------------------------------------------------------------
inline double w3j(int j1, int j2, int j3, int m1, int m2, int m3) {
    return wig3jj(2 * j1, 2 * j2, 2 * j3, 2 * m1, 2 * m2, 2 * m3);
}

// lib_math_vector_spherical_harmonics.f90:2235-2261
inline int q_max_a(int m, int n, int k, int l) {
    return std::min(std::min(n, l), (int)std::floor((double)(n + l - std::abs(m + k)) / 2.0));
}
inline int q_max_b(int m, int n, int k, int l) {
    return std::min(std::min(n, l), (int)std::floor((double)(n + l + 1 - std::abs(m + k)) / 2.0));
}

// lib_math_vector_spherical_harmonics.f90:2283-2349 (Xu 1996 eq. 5 and eq. 61)
void ab_xu_cruzan_eq34(int m, int n, int mu, int nu, int p, bool calc_a, bool calc_b,
                       double* a, double* b) {
    double s = ((m + mu) & 1) ? -1.0 : 1.0;
    double f1 = npm_over_nmm(n, m);
    double f2 = npm_over_nmm(nu, mu);
    double w2 = w3j(n, nu, p, 0, 0, 0);
    if (calc_a) {
        double f3 = nmm_over_npm(p, m + mu);
        double w1 = w3j(n, nu, p, m, mu, -m - mu);
        *a = s * ((2 * p + 1) * std::sqrt(f1 * f2 * f3) * w1 * w2);
    } else {
        *a = 0.0;
    }
    if (calc_b) {
        double f3 = nmm_over_npm(p + 1, m + mu);
        double w1 = w3j(n, nu, p + 1, m, mu, -m - mu);
        *b = s * ((2 * p + 3) * std::sqrt(f1 * f2 * f3) * w1 * w2);
    } else {
        *b = 0.0;
    }
}

inline cd ipow(int p) {
    switch (((p % 4) + 4) % 4) {
        case 0: return cd(1, 0);
        case 1: return cd(0, 1);
        case 2: return cd(-1, 0);
        default: return cd(0, -1);
    }
}

inline int blk(int n1, int n, int m) { return n * n - n1 * n1 + (m + n); }

// Vector translation coefficients A_mn^{mu nu}, B_mn^{mu nu}
// (lib_math_vector_spherical_harmonics.f90:1354-1585).  Output layout:
// A[(blk(n1,n,m)) * cnt_nu + blk(nu1,nu,mu)], cnt_nu = (nu2+1)^2 - nu1^2.
void translation_xu(double x, double theta, double phi, int n1, int n2, int nu1, int nu2,
                    int z, cd* A, cd* B) {
    int nmaxr = std::max(n2, nu2);
    int pmax = 2 * nmaxr + 1;
    std::vector<cd> zn(pmax + 2);
    sph_z(z, x, pmax + 1, zn.data());
    std::vector<double> P((pmax + 1) * (pmax + 1));
    legendre_table(std::cos(theta), pmax, P.data());
    int cnt_nu = (nu2 + 1) * (nu2 + 1) - nu1 * nu1;
#pragma omp parallel
    {
        ensure_wig_temp(2 * (2 * pmax + 2));
#pragma omp for schedule(dynamic)
        for (int n = n1; n <= n2; ++n) {
            for (int m = -n; m <= n; ++m) {
                for (int nu = nu1; nu <= nu2; ++nu) {
                    for (int mu = -nu; mu <= nu; ++mu) {
                        int qa = q_max_a(-m, n, mu, nu);
                        int qb = q_max_b(-m, n, mu, nu);
                        int qm = std::max(qa, qb);
                        double factorial = (2 * nu + 1);
                        factorial = factorial * npm_over_nmm(n, m);
                        factorial = factorial * nmm_over_npm(nu, mu);
                        factorial = factorial / (double)(2 * n * (n + 1));
                        cd sa(0, 0), sb(0, 0);
                        for (int q = 0; q <= qm; ++q) {
                            int p = n + nu - 2 * q;
                            bool ca = (q >= 0 && q <= qa);
                            bool cb = (q >= 1 && q <= qb);
                            double a, b;
                            ab_xu_cruzan_eq34(-m, n, mu, nu, p, ca, cb, &a, &b);
                            if (ca) {
                                double br = (double)(n * (n + 1) + nu * (nu + 1) - p * (p + 1)) * a *
                                            P[p * (p + 1) + (mu - m)];
                                sa += ipow(p) * (br * zn[p]);
                            }
                            if (cb) {
                                double br = std::sqrt((std::pow((double)(p + 1), 2) - std::pow((double)(n - nu), 2)) *
                                                      (std::pow((double)(n + nu + 1), 2) - std::pow((double)(p + 1), 2))) *
                                            b * P[(p + 1) * (p + 2) + (mu - m)];
                                sb += ipow(p + 1) * (br * zn[p + 1]);
                            }
                        }
                        double ang = (mu - m) * phi;
                        cd e(std::cos(ang), std::sin(ang));
                        cd bc = factorial * e;
                        double sgn = (m & 1) ? -1.0 : 1.0;
                        int row = blk(n1, n, m), col = blk(nu1, nu, mu);
                        A[(size_t)row * cnt_nu + col] = sgn * bc * sa;
                        B[(size_t)row * cnt_nu + col] = -sgn * bc * sb;
                    }
                }
            }
        }
    }
}

// ------------------------------------------------------------------------------------------
// Mie coefficients (FoggySim/src/lib/mie_theory/lib_mie_ss_helper_functions.f90:628-722,
// logarithmic derivative 751-924, n_c 937-951)
// ------------------------------------------------------------------------------------------
int get_n_c(double x) { return (int)std::ceil(x + 4.05 * std::cbrt(x) + 2.0); }

void mie_ab(double x, cd m, int n1, int n2, cd* a_n, cd* b_n) {
    int number = n2 - n1 + 1;
    cd mx = m * x;
    int n_mx = std::max(get_n_c(std::fabs(x)), (int)std::abs(mx)) + 15;
    int n_max = n2;
    std::vector<cd> An(number);
    cd buf(0, 0);
    for (int i = n_mx; i >= n1 + 1; --i) {
        cd ndm = (double)i / mx;
        buf = ndm - 1.0 / (buf + ndm);
        if (i <= n_max + 1) An[i - 1 - n1] = buf;
    }
    std::vector<double> j(n2 + 2), y(n2 + 2);
    sph_jn(x, n2 + 1, j.data());
    sph_yn(x, n2 + 1, y.data());
    for (int i = 0; i < number; ++i) {
        int n = n1 + i;
        double ndx = (double)n / x;
        cd jn(j[n], 0), jnm(j[n - 1], 0), hn(j[n], y[n]), hnm(j[n - 1], y[n - 1]);
        cd bufa = An[i] / m + ndx;
        a_n[i] = (bufa * jn - jnm) / (bufa * hn - hnm);
        cd bufb = m * An[i] + ndx;
        b_n[i] = (bufb * jn - jnm) / (bufb * hn - hnm);
    }
}


// ------------------------------------------------------------------------------------------
// cartesian <-> spherical (libmath/src/math/lib_math_type_operator.f90:3600-3647, ISO 31-11)
// ------------------------------------------------------------------------------------------
void to_spherical(const double* c, double* rho, double* theta, double* phi) {
    double r = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
    *rho = r;
    *theta = (r == 0.0) ? 0.0 : std::acos(c[2] / r);
    *phi = (c[0] == 0.0 && c[1] == 0.0) ? 0.0 : std::atan2(c[1], c[0]);
}
void to_cartesian(double rho, double theta, double phi, double* c) {
    double rs = rho * std::sin(theta);
    c[0] = rs * std::cos(phi);
    c[1] = rs * std::sin(phi);
    c[2] = rho * std::cos(theta);
}

// ------------------------------------------------------------------------------------------
// plane-wave coefficients p_nm, q_nm (lib_mie_illumination.f90:295-354 single wave,
// 392-478 several waves with Jones vector, 636-763 core; Xu 1995 eq. 20 with erratum)
// out layout: index n*n - n1*n1 + (m+n) for n = n1..n2
// ------------------------------------------------------------------------------------------
struct Wave {
    double theta, phi, jre, jim, yre, yim, g, phase, d0[3];
};

void pq_core(double alpha, double beta, int n1, int n2, bool has_e, cd e, cd* p, cd* q) {
    std::vector<double> pi((n2 + 1) * (n2 + 1)), tau((n2 + 1) * (n2 + 1));
    pi_tau_table(alpha, n2, 0, pi.data(), tau.data());
    for (int n = n1; n <= n2; ++n) {
        double brn = 1.0 / (double)(n * (n + 1));
        for (int m = -n; m <= n; ++m) {
            int o = blk(n1, n, m);
            if (alpha == 0.0 && m != -1 && m != 1) {
                p[o] = 0.0;
                q[o] = 0.0;
                continue;
            }
            double br = -m * beta;
            cd bc = brn * cd(std::cos(br), std::sin(br));
            cd pv = tau[n * (n + 1) + m] * bc;
            cd qv = pi[n * (n + 1) + m] * bc;
            if (has_e) {
                pv = e * pv;
                qv = e * qv;
            }
            p[o] = pv;
            q[o] = qv;
        }
    }
}

void pq_single(const double* kc, const double* d, int n1, int n2, bool te, double phase, cd* p, cd* q) {
    double rho, alpha, beta;
    to_spherical(kc, &rho, &alpha, &beta);
    double dn = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    if (dn > 0.0 || phase != 0.0) {
        double dot = kc[0] * d[0] + kc[1] * d[1] + kc[2] * d[2] + phase;
        pq_core(alpha, beta, n1, n2, true, cd(std::cos(dot), std::sin(dot)), p, q);
    } else {
        pq_core(alpha, beta, n1, n2, false, cd(1, 0), p, q);
    }
    if (te) {
        int cnt = (n2 + 1) * (n2 + 1) - n1 * n1;
        for (int i = 0; i < cnt; ++i) std::swap(p[i], q[i]);
    }
}

void pq_multi(const std::vector<Wave>& waves, double lambda0, double n_medium, const double* d0j,
              int n1, int n2, cd* p, cd* q) {
    int cnt = (n2 + 1) * (n2 + 1) - n1 * n1;
    std::fill(p, p + cnt, cd(0, 0));
    std::fill(q, q + cnt, cd(0, 0));
    std::vector<cd> ta(cnt), tb(cnt), bp(cnt), bq(cnt);
    for (const Wave& w : waves) {
        double d[3] = {d0j[0] - w.d0[0], d0j[1] - w.d0[1], d0j[2] - w.d0[2]};
        double kc[3];
        to_cartesian(2.0 * PI * n_medium / lambda0, w.theta, w.phi, kc);
        std::fill(bp.begin(), bp.end(), cd(0, 0));
        std::fill(bq.begin(), bq.end(), cd(0, 0));
        double ax = std::abs(cd(w.jre, w.jim));
        double gx = std::atan2(w.jim, w.jre) + w.phase;
        if (ax > 0) {
            pq_single(kc, d, n1, n2, false, gx, ta.data(), tb.data());
            for (int i = 0; i < cnt; ++i) { bp[i] = ax * ta[i]; bq[i] = ax * tb[i]; }
        }
        double ay = std::abs(cd(w.yre, w.yim));
        double gy = std::atan2(w.yim, w.yre) + w.phase;
        if (ay > 0) {
            pq_single(kc, d, n1, n2, true, gy, ta.data(), tb.data());
            for (int i = 0; i < cnt; ++i) { bp[i] += ay * ta[i]; bq[i] += ay * tb[i]; }
        }
        for (int i = 0; i < cnt; ++i) { p[i] += w.g * bp[i]; q[i] += w.g * bq[i]; }
    }
}

// ------------------------------------------------------------------------------------------
// libtree universal index (libtree/src/lib/lib_tree_helper_functions.f90:202-364, 532-614,
// 1204-1266) and scaling (libtree/src/lib/lib_tree.f90:320-374)
// ------------------------------------------------------------------------------------------
uint64_t coordinate_binary(double f) {
    uint64_t bits;
    std::memcpy(&bits, &f, 8);
    int64_t e = (int64_t)(bits >> 52);               // sign bit is zero for f >= 0
    uint64_t mant = (bits << 11) | (1ull << 63);
    int64_t shift = 1023 - e - 1;
    if (shift >= 64) return 0;                      // gfortran ishft beyond the width
    if (shift <= 0) return mant;                    // f >= 1 does not occur after scaling
    return mant >> shift;
}

// 192 interleaved bits, dimension 1 most significant in each 3-bit group; the universal
// index at level l is the top 3*l bits of the top 64 interleaved bits.
int64_t universal_index(const double* pt, int l) {
    uint64_t cb[3] = {coordinate_binary(pt[0]), coordinate_binary(pt[1]), coordinate_binary(pt[2])};
    uint64_t top = 0;   // top 64 interleaved bits: coordinate bits 63..42 (22 groups, 66 bits)
    int pos = 63;
    for (int b = 63; b >= 0 && pos >= 0; --b) {
        for (int d = 0; d < 3 && pos >= 0; ++d) {
            if ((cb[d] >> b) & 1ull) top |= (1ull << pos);
            --pos;
        }
    }
    int nbits = 3 * l;
    if (nbits >= 64) return (int64_t)top;
    return (int64_t)(top >> (64 - nbits));
}

void scale_points(int n, const double* c, double* out, double* D_out, double* xmin_out) {
    double xmin[3], xmax[3], D[3];
    for (int d = 0; d < 3; ++d) {
        xmin[d] = c[d];
        xmax[d] = c[d];
        for (int i = 1; i < n; ++i) {
            xmin[d] = std::min(xmin[d], c[3 * i + d]);
            xmax[d] = std::max(xmax[d], c[3 * i + d]);
        }
        D[d] = (xmax[d] - xmin[d]) * (1.0 + std::ldexp(1.0, -52));
    }
    double Dm = std::max(D[0], std::max(D[1], D[2]));
    for (int i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d)
            out[3 * i + d] = (Dm > 0) ? (c[3 * i + d] - xmin[d]) / Dm : 0.0;
    if (D_out) *D_out = Dm;
    if (xmin_out) for (int d = 0; d < 3; ++d) xmin_out[d] = xmin[d];
}

// ------------------------------------------------------------------------------------------
// the multi-sphere problem (FoggySim/src/lib/mie_theory/lib_mie_type.f90:43-99)

// ------------------------------------------------------------------------------------------
// Gaussian beams in the plane-wave approximation (lib_mie_illumination.f90:781-918 case 3,
// 1022-1050; lib_field_gaussian_beam.f90:111-891).  The localised-approximation branches of the
// reference (cases 1 and 2) are commented out there and have no restatement.
// ------------------------------------------------------------------------------------------
// lib_math_get_matrix_rot, Euler x-convention (lib_math_type_operator.f90:1768-1810)
void rot3(double phi, double theta, double psi, double R[9]) {
    const double cph = std::cos(phi), sph = std::sin(phi), cth = std::cos(theta), sth = std::sin(theta);
    const double cps = std::cos(psi), sps = std::sin(psi);
    R[0] = cps * cph - cth * sph * sps;  R[1] = cps * sph + cth * cph * sps;  R[2] = sps * sth;
    R[3] = -sps * cph - cth * sph * cps; R[4] = -sps * sph + cth * cph * cps; R[5] = cps * sth;
    R[6] = sth * sph;                    R[7] = -sth * cph;                   R[8] = cth;
}
void mul3(const double R[9], const double v[3], double o[3]) {
    const double a = v[0], b = v[1], c = v[2];
    o[0] = R[0] * a + R[1] * b + R[2] * c;
    o[1] = R[3] * a + R[4] * b + R[5] * c;
    o[2] = R[6] * a + R[7] * b + R[8] * c;
}
// physicists' Hermite polynomial H_n (lib_math_hermite.f90:93-127): H_0 = 1, H_1 = 2x,
// H_{k+1} = 2x H_k - 2k H_{k-1}
double hermite(int n, double x) {
    double h0 = 1.0, h1 = 2.0 * x;
    if (n == 0) return h0;
    for (int k = 1; k < n; ++k) {
        const double h2 = 2.0 * x * h1 - 2.0 * k * h0;
        h0 = h1;
        h1 = h2;
    }
    return h1;
}
double factorial(int n) {
    double f = 1.0;
    for (int i = 2; i <= n; ++i) f *= i;
    return f;
}
struct GBeam {
    double e0, lambda0, n_medium, phase, wx0, wy0;
    int tem_m, tem_n;
    cd jx, jy;
    double theta, phi;
    int convention;
    double g, d0[3];
};
// lib_field_gaussian_beam_rayleigh_length / _waist / _curvature (:817-891)
double gb_zr(double w0, const GBeam& b) { return PI * w0 * w0 * b.n_medium / b.lambda0; }
double gb_w(double w0, double zr, double z) { return w0 * std::sqrt(1.0 + (z / zr) * (z / zr)); }
double gb_c(double zr, double z) { return z / (z * z + zr * zr); }
bool gb_rotated(const GBeam& b) { return b.phi != 0.0 || b.theta != 0.0; }
// world point relative to the beam origin -> beam frame (:127-133)
void gb_to_beam(const GBeam& b, const double x[3], double o[3]) {
    if (gb_rotated(b)) {
        double R[9];
        rot3(PI / 2.0 + b.phi, b.theta, PI / 2.0 + b.phi, R);
        mul3(R, x, o);
    } else {
        o[0] = x[0]; o[1] = x[1]; o[2] = x[2];
    }
}
// lib_fiel_gaussian_beam_hermite_scalar (:401-507) at a beam-frame point
cd gb_scalar(const GBeam& b, const double x[3]) {
    const double k = 2.0 * PI * b.n_medium / b.lambda0;
    const double zrx = gb_zr(b.wx0, b), wx = gb_w(b.wx0, zrx, x[2]), crx = gb_c(zrx, x[2]);
    const double zry = gb_zr(b.wy0, b), wy = gb_w(b.wy0, zry, x[2]), cry = gb_c(zry, x[2]);
    const double hx = hermite(b.tem_m, x[0] * std::sqrt(2.0) / wx), hy = hermite(b.tem_n, x[1] * std::sqrt(2.0) / wy);
    cd c = std::sqrt(b.wx0 / wx) * hx * std::exp(-x[0] * x[0] / (wx * wx)) *
           std::exp(cd(0, -k * x[0] * x[0] * crx / 2.0));
    c = std::sqrt(b.wy0 / wy) * hy * std::exp(-x[1] * x[1] / (wy * wy)) * std::exp(cd(0, -k * x[1] * x[1] * cry / 2.0)) * c;
    const double amp = b.e0 * std::sqrt(1.0 / (std::pow(2.0, b.tem_m + b.tem_n) * factorial(b.tem_m) *
                                               factorial(b.tem_n) * PI));
    c = amp * std::exp(cd(0, -k * x[2] + b.phase)) * c;
    c = std::exp(cd(0, (b.tem_m + 0.5) * std::atan2(x[2], zrx) + (b.tem_n + 0.5) * std::atan2(x[2], zry))) * c;
    return b.convention == 2 ? std::conj(c) : c;
}
// get_derivative_xy (:573-595), get_derivative_z (:597-679)
double gb_dxy(const GBeam& b, double w0, double xy, double z) {
    if (xy == 0.0 || z == 0.0) return 0.0;
    return -2.0 * PI * b.lambda0 * xy * z * b.n_medium /
           ((PI * b.n_medium) * (PI * b.n_medium) * std::pow(w0, 4.0) + (b.lambda0 * z) * (b.lambda0 * z));
}
double gb_dz(const GBeam& b, double x, double y, double z) {
    const double pn2 = (PI * b.n_medium) * (PI * b.n_medium), lz2 = (b.lambda0 * z) * (b.lambda0 * z);
    const double wx2 = b.wx0 * b.wx0, wx4 = wx2 * wx2, wy2 = b.wy0 * b.wy0, wy4 = wy2 * wy2;
    double rv = (2.0 * b.tem_m * wx2 + 2.0 * x * x) / (pn2 * wx4 + lz2);
    rv += (2.0 * b.tem_n * wy2 + 2.0 * y * y) / (pn2 * wy4 + lz2);
    rv += -4.0 * pn2 * x * x * wx4 / ((pn2 * wx4 + lz2) * (pn2 * wx4 + lz2));
    rv += -4.0 * pn2 * y * y * wy4 / ((pn2 * wy4 + lz2) * (pn2 * wy4 + lz2));
    rv = rv * b.lambda0 * b.lambda0 / 2.0 - 2.0;
    return PI * b.n_medium * rv / b.lambda0;
}
// lib_field_gaussian_beam_hermite_get_propagation_direction (:191-225, :546-571), world frame
void gb_direction(const GBeam& b, const double xw[3], double kv[3]) {
    double x[3];
    gb_to_beam(b, xw, x);
    double k[3] = {-gb_dxy(b, b.wx0, x[0], x[2]), -gb_dxy(b, b.wy0, x[1], x[2]), -gb_dz(b, x[0], x[1], x[2])};
    const double a = std::sqrt(k[0] * k[0] + k[1] * k[1] + k[2] * k[2]);
    for (double& v : k) v /= a;
    if (gb_rotated(b)) {
        double R[9];
        rot3(-PI / 2.0 - b.phi, -b.theta, -PI / 2.0 - b.phi, R);
        mul3(R, k, kv);
    } else {
        kv[0] = k[0]; kv[1] = k[1]; kv[2] = k[2];
    }
}
// get_absolute_value_and_argument (:681-799) at a beam-frame point
void gb_abs_arg(const GBeam& b, const double x[3], double* absolute, double* argument) {
    const double k = 2.0 * PI * b.n_medium / b.lambda0;
    const double kz = std::fmod(k * x[2], 2.0 * PI);
    const double zrx = gb_zr(b.wx0, b), zry = gb_zr(b.wy0, b);
    const double wx = gb_w(b.wx0, zrx, x[2]), wy = gb_w(b.wy0, zry, x[2]);
    const double crx = gb_c(zrx, x[2]), cry = gb_c(zry, x[2]);
    double arg = -std::fmod(k * crx * x[0] * x[0] / 2.0, 2.0 * PI);
    arg = arg - std::fmod(k * cry * x[1] * x[1] / 2.0, 2.0 * PI);
    arg = arg - kz + b.phase;
    arg = arg + (b.tem_m + 0.5) * std::atan2(x[2], zrx);
    arg = arg + (b.tem_n + 0.5) * std::atan2(x[2], zry);
    const double hx = hermite(b.tem_m, x[0] * std::sqrt(2.0) / wx), hy = hermite(b.tem_n, x[1] * std::sqrt(2.0) / wy);
    if (hx * hy < 0.0) arg = arg - PI;
    arg = std::fmod(arg, 2.0 * PI);
    if (b.convention == 2) arg = -arg;
    if (arg < 0.0) arg = 2.0 * PI + arg;
    *argument = arg;
    const double a = std::sqrt(b.wx0 / wx) * hx * std::exp(-(x[0] / wx) * (x[0] / wx)) * std::sqrt(b.wy0 / wy) * hy *
                     std::exp(-(x[1] / wy) * (x[1] / wy)) * b.e0 *
                     std::sqrt(1.0 / ((double)(1 << (b.tem_m + b.tem_n)) * factorial(b.tem_m) * factorial(b.tem_n) * PI));
    *absolute = std::fabs(a);
}
// lib_field_gaussian_beam_hermite_get_plane_wave_approximation (:256-358): the plane wave that
// stands in for the beam at world point xw (relative to the beam origin); its amplitude is
// returned but, as in the reference, not used by the plane-wave coefficients
Wave gb_plane_wave(const GBeam& b, const double xw[3], double* amplitude) {
    double x[3], kv[3], rho, th, ph;
    gb_to_beam(b, xw, x);
    gb_direction(b, xw, kv);
    to_spherical(kv, &rho, &th, &ph);
    double absolute, argument;
    gb_abs_arg(b, x, &absolute, &argument);
    double phase = argument + std::fmod(2.0 * PI * x[2] / b.lambda0, 2.0 * PI);
    phase = std::fmod(phase, 2.0 * PI);
    if (phase < 0.0) phase = 2.0 * PI + phase;
    double ax[3] = {1, 0, 0}, ay[3] = {0, 1, 0};
    if (ph != 0.0 || th != 0.0) {
        double R[9], t[3];
        rot3(PI / 2.0 + b.phi, b.theta, PI / 2.0 + b.phi, R);
        mul3(R, ax, t); ax[0] = t[0]; ax[1] = t[1]; ax[2] = t[2];
        mul3(R, ay, t); ay[0] = t[0]; ay[1] = t[1]; ay[2] = t[2];
    }
    cd px = b.jx * std::fabs(ax[0]) + b.jy * std::fabs(ay[0]);
    cd py = b.jy * std::fabs(ay[1]) + b.jx * std::fabs(ax[1]);
    const double nrm = std::sqrt(std::norm(px) + std::norm(py));
    px /= nrm;
    py /= nrm;
    Wave w;
    w.theta = th;
    w.phi = ph;
    w.jre = px.real(); w.jim = px.imag();
    w.yre = py.real(); w.yim = py.imag();
    // case 3 scales by g twice: once as the plane wave's own g, once per beam (:864-877)
    w.g = b.g * b.g;
    w.phase = phase;
    for (int d = 0; d < 3; ++d) w.d0[d] = b.d0[d];
    if (amplitude) *amplitude = absolute;
    return w;
}
// ------------------------------------------------------------------------------------------
struct Problem {
    double lambda0, n_medium, k;
    int n1, n2, z, row_rule;
    int N, NP;
    std::vector<double> centres;
    std::vector<int> pidx;
    std::vector<cd> mref;
    std::vector<double> radius;
    std::vector<int> nr;
    std::vector<std::vector<cd>> an, bn;   // per parameter, index n - nr1
    std::vector<Wave> waves;
    std::vector<GBeam> beams;
    int cnt() const { return (n2 + 1) * (n2 + 1) - n1 * n1; }
    // cache of translation blocks per ordered pair (geometry only, bit-identical to recomputing)
    std::vector<std::vector<cd>> cacheA, cacheB;
    std::vector<char> cached;
};

void sphere_range(const Problem& P, int j, int* a, int* b) {
    int ip = P.pidx[j];
    *a = std::max(P.nr[2 * ip], P.n1);
    *b = std::min(P.nr[2 * ip + 1], P.n2);
}

// lib_mie_ms_solver_get_vector_b_all (lib_mie_ms_solver_interface.f90:230-315); the
// product a_n * p_nm runs over the intersection of the degree ranges
// (lib_math_type_operator.f90:3489-3516), entries outside stay zero.
void vector_b(const Problem& P, cd* b, cd* pq_out) {
    int C = P.cnt();
    std::vector<cd> p(C), q(C);
    std::vector<cd> pb(C), qb(C);
    for (int j = 0; j < P.N; ++j) {
        pq_multi(P.waves, P.lambda0, P.n_medium, &P.centres[3 * j], P.n1, P.n2, p.data(), q.data());
        // Gaussian beams: each sphere sees its own local plane wave (lib_mie_illumination.f90:232-247)
        for (const GBeam& b : P.beams) {
            const double xw[3] = {P.centres[3 * j] - b.d0[0], P.centres[3 * j + 1] - b.d0[1],
                                  P.centres[3 * j + 2] - b.d0[2]};
            std::vector<Wave> one{gb_plane_wave(b, xw, nullptr)};
            pq_multi(one, P.lambda0, P.n_medium, &P.centres[3 * j], P.n1, P.n2, pb.data(), qb.data());
            for (int i = 0; i < C; ++i) {
                p[i] += pb[i];
                q[i] += qb[i];
            }
        }
        int ip = P.pidx[j];
        int a0 = P.nr[2 * ip];
        int ja, jb;
        sphere_range(P, j, &ja, &jb);
        cd* bj = b + (size_t)2 * C * j;
        for (int i = 0; i < 2 * C; ++i) bj[i] = 0.0;
        for (int n = ja; n <= jb; ++n)
            for (int m = -n; m <= n; ++m) {
                int o = blk(P.n1, n, m);
                bj[o] = P.an[ip][n - a0] * p[o];
                bj[C + o] = P.bn[ip][n - a0] * q[o];
            }
        if (pq_out) {
            for (int i = 0; i < C; ++i) {
                pq_out[(size_t)2 * C * j + i] = p[i];
                pq_out[(size_t)2 * C * j + C + i] = q[i];
            }
        }
    }
}

// Direct operator y = A x (lib_mie_ms_solver_calculate_vector_b_without_transposed_all,
// lib_mie_ms_solver_interface.f90:806-998), rows of target spheres j0 <= j < j1.  With
// cache = false the translation blocks are recomputed on every call, as the reference does.
void matvec_direct(Problem& P, const cd* x, cd* y, int j0 = 0, int j1 = -1, bool cache = true) {
    int C = P.cnt();
    int N = P.N;
    if (j1 < 0) j1 = N;
    if (cache && P.cached.size() != (size_t)N * N) {
        P.cached.assign((size_t)N * N, 0);
        P.cacheA.assign((size_t)N * N, {});
        P.cacheB.assign((size_t)N * N, {});
    }
    for (size_t i = (size_t)2 * C * j0; i < (size_t)2 * C * j1; ++i) y[i] = 0.0;
    // parallel over (target, source) blocks of rows, as the reference's OMP loop over j
    std::vector<std::pair<int, int>> work;
    for (int j = j0; j < j1; ++j) work.push_back({j, 0});
#pragma omp parallel for schedule(dynamic)
    for (int w = 0; w < (int)work.size(); ++w) {
        int j = work[w].first;
        std::vector<cd> lA, lB;
        ensure_wig_temp(2 * (4 * P.n2 + 8));
        int ip = P.pidx[j];
        int a0 = P.nr[2 * ip];
        cd* yj = y + (size_t)2 * C * j;
        for (int l = 0; l < N; ++l) {
            if (l == j) {
                for (int i = 0; i < 2 * C; ++i) yj[i] += x[(size_t)2 * C * j + i];
                continue;
            }
            int ja, jb, la, lb;
            sphere_range(P, j, &ja, &jb);
            sphere_range(P, l, &la, &lb);
            // rows are zero unless the sphere's own range covers the global range
            bool rows = !(P.row_rule) || (P.n2 <= jb && P.n1 >= ja);
            if (!rows) continue;
            int cj = (jb + 1) * (jb + 1) - ja * ja;
            int cl = (lb + 1) * (lb + 1) - la * la;
            size_t key = (size_t)j * N + l;
            const cd* A;
            const cd* B;
            if (!cache || !P.cached[key]) {
                double kd[3];
                for (int d = 0; d < 3; ++d) kd[d] = P.k * (P.centres[3 * l + d] - P.centres[3 * j + d]);
                double rho, th, ph;
                to_spherical(kd, &rho, &th, &ph);
                lA.resize((size_t)cj * cl);
                lB.resize((size_t)cj * cl);
                translation_xu(rho, th, ph, ja, jb, la, lb, P.z, lA.data(), lB.data());
                if (cache) {
                    P.cacheA[key] = lA;
                    P.cacheB[key] = lB;
                    P.cached[key] = 1;
                }
            }
            if (cache) {
                A = P.cacheA[key].data();
                B = P.cacheB[key].data();
            } else {
                A = lA.data();
                B = lB.data();
            }
            const cd* xa = x + (size_t)2 * C * l;
            const cd* xb = xa + C;
            for (int n = ja; n <= jb; ++n) {
                cd an = P.an[ip][n - a0], bn = P.bn[ip][n - a0];
                for (int m = -n; m <= n; ++m) {
                    int row = blk(ja, n, m);
                    cd s1(0, 0), s2(0, 0);
                    for (int nu = la; nu <= lb; ++nu)
                        for (int mu = -nu; mu <= nu; ++mu) {
                            int col = blk(la, nu, mu);
                            int xo = blk(P.n1, nu, mu);
                            cd a = A[(size_t)row * cl + col], bb = B[(size_t)row * cl + col];
                            s1 += a * xa[xo] + bb * xb[xo];
                            s2 += bb * xa[xo] + a * xb[xo];
                        }
                    int o = blk(P.n1, n, m);
                    yj[o] += an * s1;
                    yj[C + o] += bn * s2;
                }
            }
        }
    }
}

// Restarted GMRES with modified Gram-Schmidt and Givens rotations (Saad & Schultz 1986), the
// method of the CERFACS package the reference drives (lib_solver_GMRES.f90:116-316; the
// package itself is not in the reference tree).  Inner products may carry a diagonal weight
// w (w = 1: the reference's raw coefficient basis).  Stops when ||b - A x||_w / ||b||_w <= tol,
// with the residual recomputed explicitly at each restart.
struct GmresOut { int iterations, restarts, matvecs, status; double backward_error; };

template <class Op>
GmresOut gmres(Op op, size_t n, const cd* b, cd* x, int restart, double tol, int maxit,
               const double* w) {
    auto dot = [&](const cd* u, const cd* v) {
        cd s(0, 0);
        for (size_t i = 0; i < n; ++i) s += std::conj(u[i]) * v[i] * (w ? w[i] : 1.0);
        return s;
    };
    auto nrm = [&](const cd* u) { return std::sqrt(std::real(dot(u, u))); };
    GmresOut o{0, 0, 0, 0, 0.0};
    std::vector<cd> r(n), tmp(n);
    double bnorm = nrm(b);
    if (bnorm == 0.0) {
        for (size_t i = 0; i < n; ++i) x[i] = 0.0;
        return o;
    }
    std::vector<std::vector<cd>> V(restart + 1, std::vector<cd>(n));
    std::vector<cd> H((size_t)(restart + 1) * restart), g(restart + 1), cs(restart), sn(restart);
    auto residual = [&]() {
        op(x, tmp.data());
        o.matvecs++;
        for (size_t i = 0; i < n; ++i) r[i] = b[i] - tmp[i];
        return nrm(r.data());
    };
    double beta = residual();
    o.backward_error = beta / bnorm;
    while (o.backward_error > tol && o.iterations < maxit) {
        for (size_t i = 0; i < n; ++i) V[0][i] = r[i] / beta;
        std::fill(g.begin(), g.end(), cd(0, 0));
        g[0] = beta;
        int k = 0;
        for (; k < restart && o.iterations < maxit; ++k) {
            op(V[k].data(), V[k + 1].data());
            o.matvecs++;
            o.iterations++;
            for (int i = 0; i <= k; ++i) {
                cd h = dot(V[i].data(), V[k + 1].data());
                H[(size_t)i * restart + k] = h;
                for (size_t t = 0; t < n; ++t) V[k + 1][t] -= h * V[i][t];
            }
            double hn = nrm(V[k + 1].data());
            H[(size_t)(k + 1) * restart + k] = hn;
            for (int i = 0; i < k; ++i) {
                cd a = H[(size_t)i * restart + k], bb = H[(size_t)(i + 1) * restart + k];
                H[(size_t)i * restart + k] = std::conj(cs[i]) * a + std::conj(sn[i]) * bb;
                H[(size_t)(i + 1) * restart + k] = -sn[i] * a + cs[i] * bb;
            }
            cd a = H[(size_t)k * restart + k];
            double den = std::sqrt(std::norm(a) + hn * hn);
            if (den == 0.0) { o.status = -6; break; }
            cs[k] = a / den;
            sn[k] = hn / den;
            H[(size_t)k * restart + k] = den;
            H[(size_t)(k + 1) * restart + k] = 0.0;
            g[k + 1] = -sn[k] * g[k];
            g[k] = std::conj(cs[k]) * g[k];
            if (hn != 0.0)
                for (size_t t = 0; t < n; ++t) V[k + 1][t] /= hn;
            if (std::abs(g[k + 1]) / bnorm <= tol || hn == 0.0) { ++k; break; }
        }
        std::vector<cd> yv(k);
        for (int i = k - 1; i >= 0; --i) {
            cd s = g[i];
            for (int t = i + 1; t < k; ++t) s -= H[(size_t)i * restart + t] * yv[t];
            yv[i] = s / H[(size_t)i * restart + i];
        }
        for (int i = 0; i < k; ++i)
            for (size_t t = 0; t < n; ++t) x[t] += yv[i] * V[i][t];
        o.restarts++;
        beta = residual();
        o.backward_error = beta / bnorm;
        if (!std::isfinite(beta)) { o.status = -7; return o; }
        if (o.status == -6) return o;
    }
    if (o.backward_error > tol) o.status = -5;
    return o;
}

}  // namespace

// ==========================================================================================
// C API used by tests/ (through ctypes), __graft_entry__.smoke() and bench.py's CPU baseline
// ==========================================================================================
extern "C" {

void orc_init(int max_n) {
    int two_j = 2 * (4 * max_n + 8);
    wig_table_init(two_j, 3);
    ensure_wig_temp(two_j);
}

int orc_sph_jn(double x, int nmax, double* out) { sph_jn(x, nmax, out); return 0; }
int orc_sph_yn(double x, int nmax, double* out) { sph_yn(x, nmax, out); return 0; }
int orc_legendre_table(double x, int nmax, double* P) { legendre_table(x, nmax, P); return 0; }
int orc_pi_tau(double theta, int nmax, int cs, double* pi, double* tau) {
    pi_tau_table(theta, nmax, cs, pi, tau);
    return 0;
}
double orc_wigner_3j(int j1, int j2, int j3, int m1, int m2, int m3) {
    return w3j(j1, j2, j3, m1, m2, m3);
}
int orc_ab_xu_cruzan(int m, int n, int mu, int nu, int p, double* ab) {
    ab_xu_cruzan_eq34(m, n, mu, nu, p, true, true, &ab[0], &ab[1]);
    return 0;
}
int orc_n_c(double x) { return get_n_c(x); }

int orc_mie_ab(double x, double m_re, double m_im, int n1, int n2, double* a, double* b) {
    mie_ab(x, cd(m_re, m_im), n1, n2, reinterpret_cast<cd*>(a), reinterpret_cast<cd*>(b));
    return 0;
}

int orc_translation_xu(double x, double theta, double phi, int n1, int n2, int nu1, int nu2,
                       int z, double* A, double* B) {
    translation_xu(x, theta, phi, n1, n2, nu1, nu2, z, reinterpret_cast<cd*>(A),
                   reinterpret_cast<cd*>(B));
    return 0;
}

int64_t orc_universal_index(const double* pt, int l) { return universal_index(pt, l); }
uint64_t orc_coordinate_binary(double f) { return coordinate_binary(f); }
int orc_scale_points(int n, const double* c, double* out) {
    scale_points(n, c, out, nullptr, nullptr);
    return 0;
}

// Tree of the sphere centres (libtree/src/lib/lib_tree.f90:147-270): scaling, level-21
// universal indices, ascending order (lib_tree.f90:1353-1417; the centres of non-overlapping
// spheres are distinct at level 21, so the order is unique), l_min for k = 1 (:1162-1170) and
// l_max for s elements per box (:1188-1242) unless l_max_fixed > 0.
int orc_build_tree(int n, const double* centres, int s, int l_max_fixed, int64_t* uindex_lmax,
                   int* order, int* l_min, int* l_max) {
    std::vector<double> sc(3 * (size_t)n);
    scale_points(n, centres, sc.data(), nullptr, nullptr);
    std::vector<int64_t> u21(n);
    for (int i = 0; i < n; ++i) u21[i] = universal_index(&sc[3 * (size_t)i], 21);
    std::vector<int> ord(n);
    for (int i = 0; i < n; ++i) ord[i] = i;
    std::sort(ord.begin(), ord.end(), [&](int a, int b) { return u21[a] < u21[b]; });
    int lm = 1;
    if (l_max_fixed > 0) {
        lm = l_max_fixed;
    } else {
        for (int i = 0; i + s < n; ++i) {
            int64_t a = u21[ord[i]], b = u21[ord[i + s]];
            for (int j = 21; j >= 0; --j) {
                a >>= 3;
                b >>= 3;
                if (a == b) { lm = std::max(lm, j); break; }
            }
        }
    }
    if (l_min) *l_min = (int)(1 + std::floor(std::log((float)(1 + 1)) / std::log(2.0f)));
    if (l_max) *l_max = lm;
    if (order) for (int i = 0; i < n; ++i) order[i] = ord[i];
    if (uindex_lmax)
        for (int i = 0; i < n; ++i) uindex_lmax[i] = u21[i] >> (3 * (21 - lm));
    return 0;
}


}  // extern "C"

// ------------------------------------------------------------------------------------------
// Field at observation points (lib_mie_ms_get_field, FoggySim/src/lib/mie_theory/
// lib_mie_multi_sphere.f90:379-434, per sphere lib_mie_ss_get_field,
// lib_mie_single_sphere.f90:1397-1582) with the vector spherical wave functions of
// lib_math_vector_spherical_harmonics_components_real_xu
// (libmath/src/math/lib_math_vector_spherical_harmonics.f90:132-419):
//   M_nm = (0, i pi_nm z_n, -tau_nm z_n) e^{im phi}
//   N_nm = (n(n+1) P_n^m z_n / rho, tau_nm xi_n'/rho, i pi_nm xi_n'/rho) e^{im phi},
// rho = k r, xi_n = rho z_n, xi_n' = (xi_{n-1} + z_n - xi_{n+1}) / 2 (lib_math_bessel.f90:2115-2143),
// Legendre functions without the Condon-Shortley phase.  Components (rho, theta, phi).
// ------------------------------------------------------------------------------------------
void vswf(double theta, double phi, double r, double k, int nmax, int z, cd* M, cd* N) {
    double rho = k * r;
    std::vector<cd> zn(nmax + 2);
    sph_z(z, rho, nmax + 1, zn.data());
    std::vector<double> pi((nmax + 1) * (nmax + 1)), tau((nmax + 1) * (nmax + 1)), P((nmax + 1) * (nmax + 1));
    pi_tau_table(theta, nmax, 0, pi.data(), tau.data());
    legendre_table(std::cos(theta), nmax, P.data());
    for (int n = 1; n <= nmax; ++n) {
        cd xid = (rho * zn[n - 1] + zn[n] - rho * zn[n + 1]) / 2.0;
        for (int m = -n; m <= n; ++m) {
            int t = n * (n + 1) + m;
            cd e(std::cos(m * phi), std::sin(m * phi));
            size_t o = 3 * (size_t)(n * n - 1 + n + m);
            M[o + 0] = 0.0;
            M[o + 1] = cd(0.0, pi[t]) * zn[n] * e;
            M[o + 2] = -tau[t] * zn[n] * e;
            N[o + 0] = (double)(n * (n + 1)) * P[t] / rho * zn[n] * e;
            N[o + 1] = tau[t] * (xid * e / rho);
            N[o + 2] = cd(0.0, pi[t]) * (xid * e / rho);
        }
    }
}

// E and H of the scattered field of all spheres at one point (zero inside any sphere); the
// coefficients x in the reference layout, the global degree range for every sphere.
void field_at(const Problem& P, const cd* x, const double* pt, double e0, cd* E, cd* H) {
    const double c0 = 299792458.0;
    for (int c = 0; c < 3; ++c) E[c] = H[c] = 0.0;
    int C = P.cnt();
    int nmax = P.n2;
    std::vector<cd> M(3 * (size_t)C), N(3 * (size_t)C);
    for (int j = 0; j < P.N; ++j) {
        double d[3];
        for (int c = 0; c < 3; ++c) d[c] = pt[c] - P.centres[3 * j + c];
        double r, th, ph;
        to_spherical(d, &r, &th, &ph);
        if (!(r > P.radius[P.pidx[j]])) {
            for (int c = 0; c < 3; ++c) E[c] = H[c] = 0.0;
            return;
        }
        if (!(e0 > 1e-200)) continue;
        vswf(th, ph, r, P.k, nmax, 3, M.data(), N.data());
        const cd* a = x + (size_t)2 * C * j;
        const cd* b = a + C;
        cd es[3] = {0.0, 0.0, 0.0}, hs[3] = {0.0, 0.0, 0.0};
        for (int n = 1; n <= nmax; ++n) {
            cd en[3] = {0.0, 0.0, 0.0}, hn[3] = {0.0, 0.0, 0.0};
            for (int m = -n; m <= n; ++m) {
                int o = blk(P.n1, n, m);
                cd f = std::fabs(e0) * (2.0 * n + 1.0) * nmm_over_npm(n, m) * ipow(n);
                size_t q = 3 * (size_t)(n * n - 1 + n + m);
                for (int c = 0; c < 3; ++c) {
                    en[c] += cd(0.0, 1.0) * f * (a[o] * N[q + c] + b[o] * M[q + c]);
                    hn[c] += f * (b[o] * N[q + c] + a[o] * M[q + c]);
                }
            }
            for (int c = 0; c < 3; ++c) { es[c] += en[c]; hs[c] += hn[c]; }
        }
        double ct = std::cos(th), st = std::sin(th), cp = std::cos(ph), sp = std::sin(ph);
        cd ex = es[0] * (st * cp) + es[1] * (ct * cp) - es[2] * sp;
        cd ey = es[0] * (st * sp) + es[1] * (ct * sp) + es[2] * cp;
        cd ez = es[0] * ct - es[1] * st;
        cd hx = hs[0] * (st * cp) + hs[1] * (ct * cp) - hs[2] * sp;
        cd hy = hs[0] * (st * sp) + hs[1] * (ct * sp) + hs[2] * cp;
        cd hz = hs[0] * ct - hs[1] * st;
        double fh = P.n_medium / c0;
        E[0] += ex; E[1] += ey; E[2] += ez;
        H[0] += fh * hx; H[1] += fh * hy; H[2] += fh * hz;
    }
}

// ------------------------------------------------------------------------------------------
// ML-FMM operator of the reference: libmlfmm/src/lib/lib_ml_fmm.f90 (upward pass :387-640,
// downward pass :656-982, final summation :994-1204) with the Mie handles of
// FoggySim/src/lib/mie_theory/lib_mie_ms_ml_fmm_interface.f90 (get_u_B_i :259-379,
// translation_SS/SR/RR :381-595, get_u_phi_i_j :600-813, dor :825-981) and the octree of
// libtree/src/lib/lib_tree.f90 (E1 :492-609, E2 :611-724, I4 :994-1143, box centre
// lib_tree_helper_functions.f90:774-799, neighbours :914-997).
//
// convention 0 reproduces the reference as written: every translation uses the incident-wave
// radial function except the box-to-sphere one (z_translation_gt_r), the global order for all
// boxes, displacement target - source in the aggregation, M2L and box-to-sphere steps (source -
// target in M2M, L2L and the near field), and the box-to-sphere displacement unscaled as a point
// (lib_tree_get_unscaled_point of a difference adds x_min).  convention 1 is the consistent
// expansion: regular (j_n) translations for aggregation, M2M, L2L and box-to-sphere, the
// coupling's radial function for M2L and the near field, displacement source - target
// everywhere; it tends to the direct operator as the box order grows.
// ------------------------------------------------------------------------------------------
namespace fmmo {

void deinterleave(int64_t n, int l, int64_t c[3]) {
    c[0] = c[1] = c[2] = 0;
    for (int b = 0; b < l; ++b)
        for (int d = 0; d < 3; ++d) c[d] |= ((n >> (3 * b + (2 - d))) & 1) << b;
}
int64_t interleave(const int64_t c[3], int l) {
    int64_t n = 0;
    for (int b = 0; b < l; ++b)
        for (int d = 0; d < 3; ++d) n |= ((c[d] >> b) & 1) << (3 * b + (2 - d));
    return n;
}
void centre_norm(int64_t n, int l, double c[3]) {
    int64_t q[3];
    deinterleave(n, l, q);
    for (int d = 0; d < 3; ++d) c[d] = std::ldexp(1.0, -l) * ((double)q[d] + 0.5);
}
// I2: the box and its neighbours at distance 1 inside the domain (lib_tree_get_domain_i2)
std::vector<int64_t> i2(int64_t n, int l) {
    std::vector<int64_t> out{n};
    int64_t c[3], q[3];
    deinterleave(n, l, c);
    int64_t hi = ((int64_t)1 << l) - 1;
    for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dz = -1; dz <= 1; ++dz) {
                if (!dx && !dy && !dz) continue;
                q[0] = c[0] + dx, q[1] = c[1] + dy, q[2] = c[2] + dz;
                if (q[0] < 0 || q[1] < 0 || q[2] < 0 || q[0] > hi || q[1] > hi || q[2] > hi) continue;
                out.push_back(interleave(q, l));
            }
    return out;
}
// I4: children of the parent's I2 that are not in the box's own I2, ascending
std::vector<int64_t> i4(int64_t n, int l) {
    std::vector<int64_t> out;
    if (l == 0) return out;
    std::vector<int64_t> own = i2(n, l), par = i2(n >> 3, l - 1);
    std::sort(own.begin(), own.end());
    for (int64_t q : par)
        for (int c = 0; c < 8; ++c) {
            int64_t b = (q << 3) | c;
            if (!std::binary_search(own.begin(), own.end(), b)) out.push_back(b);
        }
    std::sort(out.begin(), out.end());
    return out;
}

struct Tree {
    int lmin, lmax;
    double D, xmin[3];
    std::vector<double> pn;          // normalised centres
    std::vector<int64_t> u21;
    std::vector<int> order;          // spheres by key
    std::vector<std::vector<int64_t>> boxes;   // per level (index l - lmin), ascending
    std::vector<std::map<int64_t, int>> id;
    // spheres of box n at level l (E1), in key order
    std::vector<int> e1(int64_t n, int l) const {
        std::vector<int> out;
        for (int i : order)
            if ((u21[i] >> (3 * (21 - l))) == n) out.push_back(i);
        return out;
    }
    std::vector<int> e2(int64_t n, int l) const {
        std::vector<int64_t> bs = i2(n, l);
        std::sort(bs.begin(), bs.end());
        std::vector<int> out;
        for (int64_t b : bs) {
            std::vector<int> e = e1(b, l);
            out.insert(out.end(), e.begin(), e.end());
        }
        return out;
    }
    bool exists(int64_t n, int l) const { return id[l - lmin].count(n) > 0; }
    void unscaled_centre(int64_t n, int l, double c[3]) const {
        centre_norm(n, l, c);
        for (int d = 0; d < 3; ++d) c[d] = c[d] * D + xmin[d];
    }
};

Tree build(int N, const double* centres, int s, int l_max_fixed) {
    Tree t;
    t.pn.resize(3 * (size_t)N);
    scale_points(N, centres, t.pn.data(), &t.D, t.xmin);
    t.u21.resize(N);
    for (int i = 0; i < N; ++i) t.u21[i] = universal_index(&t.pn[3 * (size_t)i], 21);
    t.order.resize(N);
    for (int i = 0; i < N; ++i) t.order[i] = i;
    std::sort(t.order.begin(), t.order.end(), [&](int a, int b) { return t.u21[a] < t.u21[b]; });
    int lm = 1;
    if (l_max_fixed > 0) {
        lm = l_max_fixed;
    } else {
        for (int i = 0; i + s < N; ++i) {
            int64_t a = t.u21[t.order[i]], b = t.u21[t.order[i + s]];
            for (int j = 21; j >= 0; --j) {
                a >>= 3;
                b >>= 3;
                if (a == b) { lm = std::max(lm, j); break; }
            }
        }
    }
    t.lmax = lm;
    t.lmin = std::min(2, lm);
    for (int l = t.lmin; l <= t.lmax; ++l) {
        std::vector<int64_t> b;
        for (int i : t.order) {
            int64_t v = t.u21[i] >> (3 * (21 - l));
            if (b.empty() || b.back() != v) b.push_back(v);
        }
        std::map<int64_t, int> m;
        for (size_t q = 0; q < b.size(); ++q) m[b[q]] = (int)q;
        t.boxes.push_back(b);
        t.id.push_back(m);
    }
    return t;
}

typedef std::vector<cd> Vec;   // reference layout from degree n1, [a | b]

// Per-level expansion orders, not in the reference (which expands every box to its global order):
// with digits > 0, the excess-bandwidth order L = kd + 1.8 digits^(2/3) (kd)^(1/3) of the level's
// box diagonal d = sqrt(3) D 2^-l, rounded up, never below the global order p_g, at most 45;
// digits = 0 gives p_g on every level.
int level_order(double k, double D, int l, double digits, int pg) {
    if (!(digits > 0.0)) return pg;
    const double kd = k * std::sqrt(3.0) * std::ldexp(D, -l);
    const double L = std::ceil(std::fma(1.8 * std::pow(digits, 2.0 / 3.0), std::cbrt(kd), kd));
    return (int)std::min(45.0, std::max((double)pg, L));
}

struct Fmm {
    Problem& P;
    int conv, zgt;
    Tree t;
    std::vector<int> Lv;   // expansion order per level (index l - lmin)
    int Cb;                // entries per part of a box vector (degrees n1..max Lv)
    std::map<std::array<double, 8>, std::pair<std::vector<cd>, std::vector<cd>>> cache;
    Fmm(Problem& p, int c, int z, const Tree& tr, double digits = 0.0) : P(p), conv(c), zgt(z), t(tr) {
        int lm = P.n2;
        for (int l = t.lmin; l <= t.lmax; ++l) {
            Lv.push_back(level_order(P.k, t.D, l, digits, P.n2));
            lm = std::max(lm, Lv.back());
        }
        Cb = (lm + 1) * (lm + 1) - P.n1 * P.n1;
    }

    // out(rows r1..r2) += T(kd; z) in(cols c1..c2); in and out in the layout from degree n1 with
    // Cin / Cout entries per part (-1: the spheres' global layout)
    void apply(const double kd[3], int z, int r1, int r2, int c1, int c2, const cd* in, cd* out,
               const std::vector<cd>* scale_a = nullptr, const std::vector<cd>* scale_b = nullptr, int a0 = 0,
               int Cin = -1, int Cout = -1) {
        if (Cin < 0) Cin = P.cnt();
        if (Cout < 0) Cout = P.cnt();
        double rho, th, ph;
        to_spherical(kd, &rho, &th, &ph);
        if (rho == 0.0) {   // coincident centres: the reference passes the coefficients through
            for (int n = std::max(r1, c1); n <= std::min(r2, c2); ++n)
                for (int m = -n; m <= n; ++m) {
                    int o = blk(P.n1, n, m);
                    out[o] += in[o];
                    out[Cout + o] += in[Cin + o];
                }
            return;
        }
        std::array<double, 8> key{kd[0], kd[1], kd[2], (double)z, (double)r1, (double)r2, (double)c1, (double)c2};
        auto it = cache.find(key);
        if (it == cache.end()) {
            int cr = (r2 + 1) * (r2 + 1) - r1 * r1, cc = (c2 + 1) * (c2 + 1) - c1 * c1;
            std::vector<cd> A((size_t)cr * cc), B((size_t)cr * cc);
            ensure_wig_temp(2 * (4 * std::max(std::max(r2, c2), P.n2) + 8));
            translation_xu(rho, th, ph, r1, r2, c1, c2, z, A.data(), B.data());
            it = cache.emplace(key, std::make_pair(std::move(A), std::move(B))).first;
        }
        const std::vector<cd>& A = it->second.first;
        const std::vector<cd>& B = it->second.second;
        int cc = (c2 + 1) * (c2 + 1) - c1 * c1;
        for (int n = r1; n <= r2; ++n)
            for (int m = -n; m <= n; ++m) {
                int row = blk(r1, n, m);
                cd s1(0, 0), s2(0, 0);
                for (int nu = c1; nu <= c2; ++nu)
                    for (int mu = -nu; mu <= nu; ++mu) {
                        int col = blk(c1, nu, mu), xo = blk(P.n1, nu, mu);
                        cd a = A[(size_t)row * cc + col], b = B[(size_t)row * cc + col];
                        s1 += a * in[xo] + b * in[Cin + xo];
                        s2 += b * in[xo] + a * in[Cin + xo];
                    }
                int o = blk(P.n1, n, m);
                if (scale_a) {
                    s1 *= (*scale_a)[n - a0];
                    s2 *= (*scale_b)[n - a0];
                }
                out[o] += s1;
                out[Cout + o] += s2;
            }
    }

    void run(const cd* x, cd* y) {
        const int C = P.cnt(), n1 = P.n1, n2 = P.n2, zi = P.z;
        const int z_reg = conv == 0 ? zi : 1, z_m2l = zi, z_dor = conv == 0 ? zgt : 1;
        const double sts = conv == 0 ? -1.0 : 1.0;   // aggregation, M2L, box-to-sphere
        const double k = P.k;
        const int nlev = t.lmax - t.lmin + 1;
        std::vector<std::vector<Vec>> Cc(nlev), Dd(nlev);
        for (int li = 0; li < nlev; ++li) {
            Cc[li].assign(t.boxes[li].size(), Vec(2 * (size_t)Cb, cd(0, 0)));
            Dd[li].assign(t.boxes[li].size(), Vec(2 * (size_t)Cb, cd(0, 0)));
        }
        auto rows_of = [&](int j, int* a, int* b) {
            sphere_range(P, j, a, b);
            return !P.row_rule || (n2 <= *b && n1 >= *a);
        };
        // upward step 1: aggregation at the leaves
        const int L = nlev - 1;
        for (size_t q = 0; q < t.boxes[L].size(); ++q) {
            int64_t nb = t.boxes[L][q];
            double cb[3];
            t.unscaled_centre(nb, t.lmax, cb);
            for (int i : t.e1(nb, t.lmax)) {
                int ia, ib;
                if (!rows_of(i, &ia, &ib)) continue;
                double kd[3];
                for (int d = 0; d < 3; ++d) kd[d] = k * sts * (P.centres[3 * i + d] - cb[d]);
                apply(kd, z_reg, n1, Lv[L], ia, ib, x + (size_t)2 * C * i, Cc[L][q].data(), nullptr, nullptr, 0, C, Cb);
            }
        }
        // upward step 2: M2M
        for (int li = L - 1; li >= 0; --li) {
            int l = t.lmin + li;
            for (size_t q = 0; q < t.boxes[li].size(); ++q) {
                int64_t nb = t.boxes[li][q];
                double cp[3];
                t.unscaled_centre(nb, l, cp);
                for (int c = 0; c < 8; ++c) {
                    int64_t ch = (nb << 3) | c;
                    auto it = t.id[li + 1].find(ch);
                    if (it == t.id[li + 1].end()) continue;
                    double cc[3], kd[3];
                    t.unscaled_centre(ch, l + 1, cc);
                    for (int d = 0; d < 3; ++d) kd[d] = k * (cc[d] - cp[d]);
                    apply(kd, z_reg, n1, Lv[li], n1, Lv[li + 1], Cc[li + 1][it->second].data(), Cc[li][q].data(),
                          nullptr, nullptr, 0, Cb, Cb);
                }
            }
        }
        // downward step 1: M2L over the interaction lists
        for (int li = 0; li < nlev; ++li) {
            int l = t.lmin + li;
            for (size_t q = 0; q < t.boxes[li].size(); ++q) {
                int64_t nb = t.boxes[li][q];
                double cb[3];
                t.unscaled_centre(nb, l, cb);
                for (int64_t s : i4(nb, l)) {
                    auto it = t.id[li].find(s);
                    if (it == t.id[li].end()) continue;
                    double cs[3], kd[3];
                    t.unscaled_centre(s, l, cs);
                    for (int d = 0; d < 3; ++d) kd[d] = k * sts * (cs[d] - cb[d]);
                    apply(kd, z_m2l, n1, Lv[li], n1, Lv[li], Cc[li][it->second].data(), Dd[li][q].data(), nullptr,
                          nullptr, 0, Cb, Cb);
                }
            }
        }
        // downward step 2: L2L
        for (int li = 1; li < nlev; ++li) {
            int l = t.lmin + li;
            for (size_t q = 0; q < t.boxes[li].size(); ++q) {
                int64_t nb = t.boxes[li][q];
                int pi = t.id[li - 1].at(nb >> 3);
                double cb[3], cp[3], kd[3];
                t.unscaled_centre(nb, l, cb);
                t.unscaled_centre(nb >> 3, l - 1, cp);
                for (int d = 0; d < 3; ++d) kd[d] = k * (cp[d] - cb[d]);
                apply(kd, z_reg, n1, Lv[li], n1, Lv[li - 1], Dd[li - 1][pi].data(), Dd[li][q].data(), nullptr,
                      nullptr, 0, Cb, Cb);
            }
        }
        // final summation: box-to-sphere and near field, y = x + a/b (...)
        for (size_t i = 0; i < (size_t)2 * C * P.N; ++i) y[i] = 0.0;
        for (size_t q = 0; q < t.boxes[L].size(); ++q) {
            int64_t nb = t.boxes[L][q];
            double cn[3], cb[3];
            centre_norm(nb, t.lmax, cn);
            t.unscaled_centre(nb, t.lmax, cb);
            std::vector<int> near = t.e2(nb, t.lmax);
            for (int j : t.e1(nb, t.lmax)) {
                cd* yj = y + (size_t)2 * C * j;
                int ja, jb;
                bool rows = rows_of(j, &ja, &jb);
                int ip = P.pidx[j], a0 = P.nr[2 * ip];
                double kd[3];
                for (int d = 0; d < 3; ++d)
                    kd[d] = conv == 0 ? k * ((t.pn[3 * (size_t)j + d] - cn[d]) * t.D + t.xmin[d])
                                      : k * (cb[d] - P.centres[3 * j + d]);
                if (rows) {
                    double r = std::sqrt(kd[0] * kd[0] + kd[1] * kd[1] + kd[2] * kd[2]);
                    if (r == 0.0) {
                        for (int i = 0; i < C; ++i) {
                            yj[i] += Dd[L][q][i];
                            yj[C + i] += Dd[L][q][Cb + i];
                        }
                    } else {
                        apply(kd, z_dor, ja, jb, n1, Lv[L], Dd[L][q].data(), yj, &P.an[ip], &P.bn[ip], a0, Cb, C);
                    }
                }
                for (int l : near) {
                    if (l == j) {
                        for (int i = 0; i < 2 * C; ++i) yj[i] += x[(size_t)2 * C * j + i];
                        continue;
                    }
                    if (!rows) continue;
                    int la, lb;
                    sphere_range(P, l, &la, &lb);
                    for (int d = 0; d < 3; ++d) kd[d] = k * (P.centres[3 * l + d] - P.centres[3 * j + d]);
                    apply(kd, zi, ja, jb, la, lb, x + (size_t)2 * C * l, yj, &P.an[ip], &P.bn[ip], a0);
                }
            }
        }
    }
};

}  // namespace fmmo

extern "C" {

// ---- problem-level API (mirrors foggy_set_spheres / foggy_set_plane_waves) ----------------
void* orc_problem_create(double lambda0, double n_medium, int n1, int n2, int z, int row_rule,
                         int N, const double* centres, const int* pidx, int NP,
                         const double* mref, const double* radius, const int* nr, int nw,
                         const double* theta, const double* phi, const double* jones,
                         const double* g, const double* phase, const double* d0i) {
    Problem* P = new Problem();
    P->lambda0 = lambda0;
    P->n_medium = n_medium;
    P->k = 2.0 * PI * n_medium / lambda0;
    P->n1 = n1;
    P->n2 = n2;
    P->z = z;
    P->row_rule = row_rule;
    P->N = N;
    P->NP = NP;
    P->centres.assign(centres, centres + 3 * (size_t)N);
    P->pidx.assign(pidx, pidx + N);
    for (int i = 0; i < NP; ++i) P->mref.push_back(cd(mref[2 * i], mref[2 * i + 1]));
    P->radius.assign(radius, radius + NP);
    P->nr.assign(nr, nr + 2 * NP);
    P->an.resize(NP);
    P->bn.resize(NP);
    for (int i = 0; i < NP; ++i) {
        // lib_mie_type_func_get_sphere_parameter (lib_mie_type_functions.f90:46-86)
        double x = 2.0 * PI * n_medium * radius[i] / lambda0;
        int a = nr[2 * i], b = nr[2 * i + 1];
        P->an[i].resize(b - a + 1);
        P->bn[i].resize(b - a + 1);
        mie_ab(x, P->mref[i] / n_medium, a, b, P->an[i].data(), P->bn[i].data());
    }
    for (int i = 0; i < nw; ++i) {
        Wave w;
        w.theta = theta[i];
        w.phi = phi[i];
        w.jre = jones[4 * i];
        w.jim = jones[4 * i + 1];
        w.yre = jones[4 * i + 2];
        w.yim = jones[4 * i + 3];
        w.g = g[i];
        w.phase = phase[i];
        for (int d = 0; d < 3; ++d) w.d0[d] = d0i[3 * i + d];
        P->waves.push_back(w);
    }
    return P;
}

void orc_problem_destroy(void* p) { delete static_cast<Problem*>(p); }

int64_t orc_vector_length(void* p) {
    Problem* P = static_cast<Problem*>(p);
    return (int64_t)2 * P->cnt() * P->N;
}

int orc_mie_of_param(void* p, int ip, double* a, double* b) {
    Problem* P = static_cast<Problem*>(p);
    for (size_t i = 0; i < P->an[ip].size(); ++i) {
        a[2 * i] = P->an[ip][i].real();
        a[2 * i + 1] = P->an[ip][i].imag();
        b[2 * i] = P->bn[ip][i].real();
        b[2 * i + 1] = P->bn[ip][i].imag();
    }
    return 0;
}

int orc_vector_b(void* p, double* b, double* pq) {
    Problem* P = static_cast<Problem*>(p);
    vector_b(*P, reinterpret_cast<cd*>(b), reinterpret_cast<cd*>(pq));
    return 0;
}

int orc_matvec(void* p, const double* x, double* y) {
    Problem* P = static_cast<Problem*>(p);
    matvec_direct(*P, reinterpret_cast<const cd*>(x), reinterpret_cast<cd*>(y));
    return 0;
}

// Contributions of an explicit list of ordered sphere pairs (target pj[i], source pl[i]) to y,
// each translation block recomputed as the reference does on every matvec
// (lib_mie_ms_solver_interface.f90:925-981).  Used to time a bounded sample of the operator.
int orc_pairs_apply(void* p, const double* xin, int npairs, const int* pj, const int* pl, double* yout) {
    Problem* P = static_cast<Problem*>(p);
    const cd* x = reinterpret_cast<const cd*>(xin);
    cd* y = reinterpret_cast<cd*>(yout);
    int C = P->cnt();
#pragma omp parallel for schedule(dynamic)
    for (int w = 0; w < npairs; ++w) {
        ensure_wig_temp(2 * (4 * P->n2 + 8));
        int j = pj[w], l = pl[w];
        if (j == l) continue;
        int ja, jb, la, lb;
        sphere_range(*P, j, &ja, &jb);
        sphere_range(*P, l, &la, &lb);
        int cj = (jb + 1) * (jb + 1) - ja * ja;
        int cl = (lb + 1) * (lb + 1) - la * la;
        double kd[3];
        for (int d = 0; d < 3; ++d) kd[d] = P->k * (P->centres[3 * l + d] - P->centres[3 * j + d]);
        double rho, th, ph;
        to_spherical(kd, &rho, &th, &ph);
        std::vector<cd> A((size_t)cj * cl), B((size_t)cj * cl);
        translation_xu(rho, th, ph, ja, jb, la, lb, P->z, A.data(), B.data());
        int ip = P->pidx[j];
        int a0 = P->nr[2 * ip];
        const cd* xa = x + (size_t)2 * C * l;
        const cd* xb = xa + C;
        cd* yj = y + (size_t)2 * C * j;
        for (int n = ja; n <= jb; ++n) {
            cd an = P->an[ip][n - a0], bn = P->bn[ip][n - a0];
            for (int m = -n; m <= n; ++m) {
                int row = blk(ja, n, m);
                cd s1(0, 0), s2(0, 0);
                for (int nu = la; nu <= lb; ++nu)
                    for (int mu = -nu; mu <= nu; ++mu) {
                        int col = blk(la, nu, mu), xo = blk(P->n1, nu, mu);
                        cd a = A[(size_t)row * cl + col], bb = B[(size_t)row * cl + col];
                        s1 += a * xa[xo] + bb * xb[xo];
                        s2 += bb * xa[xo] + a * xb[xo];
                    }
                int o = blk(P->n1, n, m);
#pragma omp critical
                {
                    yj[o] += an * s1;
                    yj[C + o] += bn * s2;
                }
            }
        }
    }
    return 0;
}

// rows of target spheres j0 <= j < j1 only; cache = 0 recomputes every translation block like
// the reference (the CPU-baseline mode)
int orc_matvec_rows(void* p, const double* x, int j0, int j1, int cache, double* y) {
    Problem* P = static_cast<Problem*>(p);
    matvec_direct(*P, reinterpret_cast<const cd*>(x), reinterpret_cast<cd*>(y), j0, j1, cache != 0);
    return 0;
}

// Solve with GMRES(restart).  weights (length of the vector, may be NULL) selects the inner
// product; x holds the initial guess on entry.  info[5] = iterations, restarts, matvecs,
// status; backward error in *berr.
int orc_solve(void* p, const double* b, double* x, int restart, double tol, int maxit,
              const double* weights, int* info, double* berr) {
    Problem* P = static_cast<Problem*>(p);
    size_t n = (size_t)2 * P->cnt() * P->N;
    GmresOut o = gmres([&](const cd* u, cd* v) { matvec_direct(*P, u, v); }, n,
                       reinterpret_cast<const cd*>(b), reinterpret_cast<cd*>(x), restart, tol,
                       maxit, weights);
    info[0] = o.iterations;
    info[1] = o.restarts;
    info[2] = o.matvecs;
    info[3] = o.status;
    *berr = o.backward_error;
    return o.status;
}

// Cluster cross-sections {C_sca, C_ext, C_abs}.  The reference has the single-sphere form
// only (lib_mie_ss_helper_functions.f90:1380-1475, weights n(n+1)(2n+1)(n-m)!/(n+m)!).  For
// a cluster: C_ext sums Re(conj(p^j) a^j + conj(q^j) b^j) over spheres with the incident
// coefficients p^j, q^j at sphere j (Xu 1997, Appl. Opt. 36, total extinction); C_abs sums
// |a^j_nm|^2 (Re(1/a^j_n) - 1) + |b^j_nm|^2 (Re(1/b^j_n) - 1) (absorption of each sphere in
// its own exciting field); C_sca = C_ext - C_abs.
int orc_cross_sections(void* p, const double* xin, double* out) {
    Problem* P = static_cast<Problem*>(p);
    const cd* x = reinterpret_cast<const cd*>(xin);
    int C = P->cnt();
    std::vector<cd> bvec((size_t)2 * C * P->N), pq((size_t)2 * C * P->N);
    vector_b(*P, bvec.data(), pq.data());
    double cext = 0.0, cabs = 0.0;
    for (int j = 0; j < P->N; ++j) {
        int ip = P->pidx[j];
        int a0 = P->nr[2 * ip];
        int ja, jb;
        sphere_range(*P, j, &ja, &jb);
        for (int n = ja; n <= jb; ++n) {
            cd an = P->an[ip][n - a0], bn = P->bn[ip][n - a0];
            double ra = (std::abs(an) > 0) ? std::real(1.0 / an) - 1.0 : 0.0;
            double rb = (std::abs(bn) > 0) ? std::real(1.0 / bn) - 1.0 : 0.0;
            for (int m = -n; m <= n; ++m) {
                int o = blk(P->n1, n, m);
                double E = (double)(n * (n + 1) * (2 * n + 1)) * nmm_over_npm(n, m);
                size_t base = (size_t)2 * C * j;
                cd a = x[base + o], b = x[base + C + o];
                cext += E * std::real(std::conj(pq[base + o]) * a + std::conj(pq[base + C + o]) * b);
                cabs += E * (std::norm(a) * ra + std::norm(b) * rb);
            }
        }
    }
    double f = 4.0 * PI / (P->k * P->k);
    out[1] = f * cext;
    out[2] = f * cabs;
    out[0] = out[1] - out[2];
    return 0;
}


// ML-FMM operator (convention 0: the reference as written; 1: consistent expansion) with
// l_max fixed (> 0) or from s_opt; x, y in the reference layout.
int orc_fmm_matvec(void* p, int l_max_fixed, int s_opt, int convention, int z_gt_r, double digits, const double* x,
                   double* y) {
    Problem* P = static_cast<Problem*>(p);
    fmmo::Tree t = fmmo::build(P->N, P->centres.data(), s_opt, l_max_fixed);
    fmmo::Fmm f(*P, convention, z_gt_r, t, digits);
    f.run(reinterpret_cast<const cd*>(x), reinterpret_cast<cd*>(y));
    return 0;
}

// Octree lists of box n at level l (lib_tree_get_domain_e1 / e2 / i4): kind 1 -> spheres of
// the box, 2 -> spheres of the box and its neighbours, 3 -> the neighbour boxes
// (lib_tree_hf_get_neighbour_all_xD), 4 -> interaction-list box indices (every candidate
// inside the domain, ascending).  Returns the count; out may be NULL.
int orc_tree_domain(int N, const double* centres, int l_max_fixed, int l, int64_t n, int kind, int64_t* out,
                    int cap) {
    fmmo::Tree t = fmmo::build(N, centres, 10, l_max_fixed > 0 ? l_max_fixed : 21);
    std::vector<int64_t> v;
    if (kind == 1) for (int i : t.e1(n, l)) v.push_back(i);
    if (kind == 2) for (int i : t.e2(n, l)) v.push_back(i);
    if (kind == 3) {   // neighbours at distance 1 inside the domain, without the box itself
        std::vector<int64_t> b = fmmo::i2(n, l);
        v.assign(b.begin() + 1, b.end());
        std::sort(v.begin(), v.end());
    }
    if (kind == 4) v = fmmo::i4(n, l);
    if (out) for (int i = 0; i < (int)v.size() && i < cap; ++i) out[i] = v[i];
    return (int)v.size();
}


// M_nm, N_nm (see vswf) for n = 1..nmax: 3 complex components per (n, m) at index n^2-1+n+m
int orc_vswf(double theta, double phi, double r, double k, int nmax, int z, double* M, double* N) {
    vswf(theta, phi, r, k, nmax, z, reinterpret_cast<cd*>(M), reinterpret_cast<cd*>(N));
    return 0;
}

// scattered E and H (3 complex each per point) of coefficient vector x at npts points
int orc_field(void* p, const double* x, int npts, const double* pts, double e0, double* E, double* H) {
    Problem* P = static_cast<Problem*>(p);
#pragma omp parallel for schedule(dynamic)
    for (int i = 0; i < npts; ++i)
        field_at(*P, reinterpret_cast<const cd*>(x), pts + 3 * (size_t)i, e0,
                 reinterpret_cast<cd*>(E) + 3 * (size_t)i, reinterpret_cast<cd*>(H) + 3 * (size_t)i);
    return 0;
}

// Gaussian beams of a problem (replace any set before); per beam: waist x0, y0, TEM m, n, theta,
// phi, Jones (re x, im x, re y, im y), g, phase, origin, convention; e_field_0 = 1 and the
// problem's wavelength and medium
int orc_set_gaussian_beams(void* p, int nb, const double* waist, const int* tem, const double* theta,
                           const double* phi, const double* jones, const double* g, const double* phase,
                           const double* d0, const int* convention) {
    Problem* P = static_cast<Problem*>(p);
    P->beams.clear();
    for (int i = 0; i < nb; ++i) {
        GBeam b;
        b.e0 = 1.0;
        b.lambda0 = P->lambda0;
        b.n_medium = P->n_medium;
        b.phase = phase ? phase[i] : 0.0;
        b.wx0 = waist[2 * i];
        b.wy0 = waist[2 * i + 1];
        b.tem_m = tem[2 * i];
        b.tem_n = tem[2 * i + 1];
        b.jx = cd(jones[4 * i], jones[4 * i + 1]);
        b.jy = cd(jones[4 * i + 2], jones[4 * i + 3]);
        b.theta = theta[i];
        b.phi = phi[i];
        b.convention = convention ? convention[i] : 1;
        b.g = g[i];
        for (int d = 0; d < 3; ++d) b.d0[d] = d0 ? d0[3 * i + d] : 0.0;
        P->beams.push_back(b);
    }
    return 0;
}

// one beam's scalar field, |E| and arg E at beam-frame points, and its local plane wave at world
// points (theta, phi, Jones x re/im, y re/im, phase, amplitude per point)
int orc_gaussian_probe(double lambda0, double n_medium, double wx0, double wy0, int tem_m, int tem_n,
                       const double* jones, double theta, double phi, double phase, int convention, int npts,
                       const double* pts, double* scalar, double* absarg, double* wave) {
    GBeam b;
    b.e0 = 1.0; b.lambda0 = lambda0; b.n_medium = n_medium; b.phase = phase; b.wx0 = wx0; b.wy0 = wy0;
    b.tem_m = tem_m; b.tem_n = tem_n; b.jx = cd(jones[0], jones[1]); b.jy = cd(jones[2], jones[3]);
    b.theta = theta; b.phi = phi; b.convention = convention; b.g = 1.0;
    b.d0[0] = b.d0[1] = b.d0[2] = 0.0;
    for (int i = 0; i < npts; ++i) {
        const double* x = pts + 3 * i;
        cd f = gb_scalar(b, x);
        scalar[2 * i] = f.real();
        scalar[2 * i + 1] = f.imag();
        gb_abs_arg(b, x, absarg + 2 * i, absarg + 2 * i + 1);
        double amp = 0.0;
        Wave w = gb_plane_wave(b, x, &amp);
        double* o = wave + 8 * i;
        o[0] = w.theta; o[1] = w.phi; o[2] = w.jre; o[3] = w.jim; o[4] = w.yre; o[5] = w.yim; o[6] = w.phase;
        o[7] = amp;
    }
    return 0;
}

}  // extern "C"
