// Host-side Wigner 3j symbols and the axial translation tables built from them.
//
// The reference evaluates every 3j symbol through wigxjpf inside its translation loop
// (libmath/src/math/lib_math_wigner.f90:45-72, lib_math_vector_spherical_harmonics.f90:
// 2283-2349).  Here the symbols are computed once per handle, for whole families at a time,
// by the three-term recurrence in j3 of Schulten & Gordon (J. Math. Phys. 16, 1961 (1975)),
// run from both ends into the classically allowed region and normalised by the sum rule
// sum_j3 (2 j3 + 1) (j1 j2 j3; m1 m2 m3)^2 = 1 (the scheme of Luscombe & Luban,
// Phys. Rev. E 57, 7274 (1998)).
//
// Axial tables.  For a translation along +z by kd the reference coefficients
// A_mn^{mu nu}, B_mn^{mu nu} (lib_math_vector_spherical_harmonics.f90:1354-1585) vanish unless
// mu = m.  In the scaled coefficient basis x_nm / g_nm with g_nm = (-1)^m sqrt((n+m)!/(n-m)!)
// all factorials cancel and
//   A(m; n, nu) = sum_{q=0}^{min(n,nu)} GA[m,n,nu,q] i^p z_p(kd),       p = n + nu - 2q
//   B(m; n, nu) = sum_{q=1}^{min(n,nu)} GB[m,n,nu,q] i^{p+1} z_{p+1}(kd)
//   GA = (-1)^m (2nu+1)/(2n(n+1)) [n(n+1)+nu(nu+1)-p(p+1)] (2p+1) (n nu p; -m m 0)(n nu p; 0 0 0)
//   GB = -(-1)^m (2nu+1)/(2n(n+1)) sqrt(((p+1)^2-(n-nu)^2)((n+nu+1)^2-(p+1)^2)) (2p+3)
//        (n nu p+1; -m m 0)(n nu p; 0 0 0)
// with A(-m) = A(m) and B(-m) = -B(m).  GA/GB are what this file produces.

#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <vector>

#include "foggy_internal.h"

namespace foggy {

// All symbols (j1 j2 j3; m1 m2 -(m1+m2)) for j3 = j3min..j3max.  Returns j3min; f is resized
// to j3max - j3min + 1.  Returns -1 if the family is empty.
int wigner3j_family(int j1, int j2, int m1, int m2, std::vector<double>& f) {
    int m3 = -(m1 + m2);
    if (std::abs(m1) > j1 || std::abs(m2) > j2) { f.clear(); return -1; }
    int jmin = std::max(std::abs(j1 - j2), std::abs(m3));
    int jmax = j1 + j2;
    if (jmin > jmax) { f.clear(); return -1; }
    int cnt = jmax - jmin + 1;
    f.assign(cnt, 0.0);
    const double J1 = j1, J2 = j2, M1 = m1, M2 = m2, M3 = m3;
    auto A = [&](double j) {
        double t = (j * j - (J1 - J2) * (J1 - J2)) * ((J1 + J2 + 1) * (J1 + J2 + 1) - j * j) * (j * j - M3 * M3);
        return t > 0 ? std::sqrt(t) : 0.0;
    };
    auto Bc = [&](double j) {
        return -(2 * j + 1) * (J1 * (J1 + 1) * M3 - J2 * (J2 + 1) * M3 - j * (j + 1) * (M2 - M1));
    };
    // m3 = 0 form divided by j (j + 1): a(j+1) f(j+1) + (2j+1)(m2-m1) f(j) + a(j) f(j-1) = 0
    auto a0 = [&](double j) {
        double t = (j * j - (J1 - J2) * (J1 - J2)) * ((J1 + J2 + 1) * (J1 + J2 + 1) - j * j);
        return t > 0 ? std::sqrt(t) : 0.0;
    };
    const bool mz = (m3 == 0);
    if (cnt == 1) {
        f[0] = 1.0;
    } else {
        // upward from jmin
        std::vector<double> up(cnt, 0.0), dn(cnt, 0.0);
        up[0] = 1.0;
        for (int i = 0; i + 1 < cnt; ++i) {
            double j = jmin + i;
            double fm = (i > 0) ? up[i - 1] : 0.0;
            double v;
            if (mz) {
                double d = a0(j + 1);
                v = (d != 0.0) ? -((2 * j + 1) * (M2 - M1) * up[i] + a0(j) * fm) / d : 0.0;
            } else {
                double d = j * A(j + 1);
                v = (d != 0.0) ? -(Bc(j) * up[i] + (j + 1) * A(j) * fm) / d : 0.0;
            }
            up[i + 1] = v;
            if (std::fabs(v) > 1e200) for (int k = 0; k <= i + 1; ++k) up[k] *= 1e-200;
        }
        // downward from jmax
        dn[cnt - 1] = 1.0;
        for (int i = cnt - 1; i >= 1; --i) {
            double j = jmin + i;
            double fp = (i + 1 < cnt) ? dn[i + 1] : 0.0;
            double v;
            if (mz) {
                double d = a0(j);
                v = (d != 0.0) ? -((2 * j + 1) * (M2 - M1) * dn[i] + a0(j + 1) * fp) / d : 0.0;
            } else {
                double d = (j + 1) * A(j);
                v = (d != 0.0) ? -(Bc(j) * dn[i] + j * A(j + 1) * fp) / d : 0.0;
            }
            dn[i - 1] = v;
            if (std::fabs(v) > 1e200) for (int k = i - 1; k < cnt; ++k) dn[k] *= 1e-200;
        }
        // classically allowed interval: the recurrence's characteristic roots are complex
        int lo = -1, hi = -1;
        for (int i = 1; i + 1 < cnt; ++i) {
            double j = jmin + i;
            double disc;
            if (mz) {
                double b = (2 * j + 1) * (M2 - M1);
                disc = b * b - 4.0 * a0(j) * a0(j + 1);
            } else {
                double b = Bc(j);
                disc = b * b - 4.0 * j * (j + 1) * A(j) * A(j + 1);
            }
            if (disc < 0) {
                if (lo < 0) lo = i;
                hi = i;
            }
        }
        int mid;
        if (lo >= 0) {
            mid = (lo + hi) / 2;
        } else {
            // no oscillatory region: meet where the upward solution peaks
            mid = 0;
            double best = -1;
            for (int i = 0; i < cnt; ++i) {
                double v = std::fabs(up[i]);
                if (v > best) { best = v; mid = i; }
            }
        }
        double num = 0, den = 0;
        for (int i = std::max(0, mid - 1); i <= std::min(cnt - 1, mid + 1); ++i) {
            num += up[i] * dn[i];
            den += dn[i] * dn[i];
        }
        double s = (den > 0) ? num / den : 0.0;
        // rescale the upward part so that the two halves meet without overflow
        double big = 0;
        for (int i = 0; i <= mid; ++i) big = std::max(big, std::fabs(up[i]));
        for (int i = mid + 1; i < cnt; ++i) big = std::max(big, std::fabs(s * dn[i]));
        double inv = (big > 0) ? 1.0 / big : 1.0;
        for (int i = 0; i < cnt; ++i) f[i] = (i <= mid) ? up[i] * inv : s * dn[i] * inv;
    }
    long double norm = 0;
    for (int i = 0; i < cnt; ++i) norm += (long double)(2 * (jmin + i) + 1) * f[i] * f[i];
    double sc = (double)(1.0L / std::sqrt(norm));
    int sgn_exp = j1 - j2 - m3;
    double want = ((sgn_exp % 2) + 2) % 2 ? -1.0 : 1.0;
    if (f[cnt - 1] * want < 0) sc = -sc;
    for (int i = 0; i < cnt; ++i) f[i] *= sc;
    return jmin;
}

double wigner3j(int j1, int j2, int j3, int m1, int m2, int m3) {
    if (m1 + m2 + m3 != 0) return 0.0;
    std::vector<double> f;
    int jmin = wigner3j_family(j1, j2, m1, m2, f);
    if (jmin < 0 || j3 < jmin || j3 > j1 + j2) return 0.0;
    return f[j3 - jmin];
}

// Axial tables for degrees 1..pmax (layout in foggy_internal.h, AxialTables).
void build_axial_tables(int pmax, AxialTables& t) {
    t.pmax = pmax;
    int S = pmax + 1;
    t.offset.assign((size_t)S * S * S, -1);
    t.ga.clear();
    t.gb.clear();
    std::vector<double> w, w0;
    for (int m = 0; m <= pmax; ++m) {
        for (int n = std::max(1, m); n <= pmax; ++n) {
            for (int nu = std::max(1, m); nu <= pmax; ++nu) {
                int qmax = std::min(n, nu);
                t.offset[((size_t)m * S + n) * S + nu] = (int32_t)t.ga.size();
                int jw = wigner3j_family(n, nu, -m, m, w);    // (n nu p; -m m 0)
                int jw0 = wigner3j_family(n, nu, 0, 0, w0);   // (n nu p; 0 0 0)
                double sgn = (m & 1) ? -1.0 : 1.0;
                double pre = sgn * (2.0 * nu + 1.0) / (2.0 * n * (n + 1.0));
                for (int q = 0; q <= qmax; ++q) {
                    int p = n + nu - 2 * q;
                    double W = (p >= jw && p <= n + nu) ? w[p - jw] : 0.0;
                    double W0 = (p >= jw0 && p <= n + nu) ? w0[p - jw0] : 0.0;
                    double ga = pre * (double)(n * (n + 1) + nu * (nu + 1) - p * (p + 1)) * (2.0 * p + 1.0) * W * W0;
                    double gb = 0.0;
                    if (q >= 1) {
                        double Wb = (p + 1 >= jw && p + 1 <= n + nu) ? w[p + 1 - jw] : 0.0;
                        double r = ((p + 1.0) * (p + 1.0) - (double)(n - nu) * (n - nu)) *
                                   ((n + nu + 1.0) * (n + nu + 1.0) - (p + 1.0) * (p + 1.0));
                        gb = -pre * std::sqrt(r > 0 ? r : 0.0) * (2.0 * p + 3.0) * Wb * W0;
                    }
                    t.ga.push_back(ga);
                    t.gb.push_back(gb);
                }
            }
        }
    }
}

// The same coefficients laid out for coalesced device reads: for each k a block of
// (pmax + 1) q-planes, each a dense W x W grid over (n, nu) in [lo, pmax]^2 (lo = max(1, k),
// W = pmax - lo + 1) of (GA, GB) pairs, zero where q > min(n, nu).  koff[k] is the block start
// in units of pairs.
void build_axial_tables_qmajor(const AxialTables& t, std::vector<int64_t>& koff, std::vector<double>& gab) {
    int pmax = t.pmax;
    int S = pmax + 1;
    koff.assign(S + 1, 0);
    int64_t tot = 0;
    for (int k = 0; k <= pmax; ++k) {
        koff[k] = tot;
        int lo = std::max(1, k);
        int W = pmax - lo + 1;
        tot += (int64_t)(pmax + 1) * W * W;
    }
    koff[S] = tot;
    gab.assign(2 * (size_t)tot, 0.0);
    for (int k = 0; k <= pmax; ++k) {
        int lo = std::max(1, k);
        int W = pmax - lo + 1;
        for (int n = lo; n <= pmax; ++n)
            for (int nu = lo; nu <= pmax; ++nu) {
                int o = t.offset[((size_t)k * S + n) * S + nu];
                int qm = std::min(n, nu);
                for (int q = 0; q <= qm; ++q) {
                    size_t d = (size_t)koff[k] + ((size_t)q * W + (n - lo)) * W + (nu - lo);
                    gab[2 * d] = t.ga[o + q];
                    gab[2 * d + 1] = t.gb[o + q];
                }
            }
    }
}

// Scalar coaxial coefficients.  With S(m; a, b) = sum_p i^p (2p+1) (a b p; -m m 0)(a b p; 0 0 0) z_p
// (p = a + b - 2q) the axial coefficients above are
//   A(m; n, nu) = pre [2 nu (nu+1) S(m;n,nu) + i kd c1 S(m;n,nu+1) - i kd c2 S(m;n,nu-1)]
//   B(m; n, nu) = pre 2 i m kd S(m;n,nu)
//   pre = (-1)^m (2nu+1)/(2n(n+1)), c1 = 2nu sqrt((nu+1)^2-m^2)/(2nu+1), c2 = 2(nu+1) sqrt(nu^2-m^2)/(2nu+1)
// (the vector-from-scalar translation relation; checked against the 3j sums to rounding).  This
// table holds (2p+1)(a b p; -m m 0)(a b p; 0 0 0) for m = 0..NM, a, b = m..NM, q = 0..min(a, b),
// q-major: koff[m] + (q W + (a - m)) W + (b - m), W = NM - m + 1.
void build_scalar_gaunt_qmajor(int NM, std::vector<int64_t>& koff, std::vector<double>& gs) {
    koff.assign(NM + 2, 0);
    int64_t tot = 0;
    for (int m = 0; m <= NM; ++m) {
        koff[m] = tot;
        int W = NM - m + 1;
        tot += (int64_t)(NM + 1) * W * W;
    }
    koff[NM + 1] = tot;
    gs.assign((size_t)tot, 0.0);
    std::vector<double> w, w0;
    for (int m = 0; m <= NM; ++m) {
        int W = NM - m + 1;
        for (int a = m; a <= NM; ++a)
            for (int b = m; b <= NM; ++b) {
                int jw = wigner3j_family(a, b, -m, m, w);
                int jw0 = wigner3j_family(a, b, 0, 0, w0);
                int qm = std::min(a, b);
                for (int q = 0; q <= qm; ++q) {
                    int p = a + b - 2 * q;
                    double W1 = (jw >= 0 && p >= jw && p <= a + b) ? w[p - jw] : 0.0;
                    double W0 = (jw0 >= 0 && p >= jw0 && p <= a + b) ? w0[p - jw0] : 0.0;
                    gs[(size_t)koff[m] + ((size_t)q * W + (a - m)) * W + (b - m)] = (2.0 * p + 1.0) * W1 * W0;
                }
            }
    }
}

// Wigner small-d at a right angle, Delta^j_{ba} = d^j_{ba}(pi/2), for j = 0..pmax and
// a, b = 0..j, stored a-major: out[delta_offset(j) + a (j + 1) + b], delta_offset(j) =
// j (j + 1)(2j + 1)/6.  Every rotation of the operator factors through it,
//   d^j_{m'm}(beta) = i^{m'-m} sum_s Delta^j_{sm'} e^{-i s beta} Delta^j_{sm},
// and the other three quadrants follow from
//   Delta_{b,-a} = (-1)^{j+b} Delta_{ba},  Delta_{-b,a} = (-1)^{j+a} Delta_{ba}.
// Each column (m' >= |m|) is run up in j by the three-term recurrence of the Jacobi polynomials
// behind d^j_{m'm}, in long double, from d^{m'}_{m'm} = (-1)^{m'-m} sqrt(C(2m', m'+m)) 2^{-m'}.
void build_delta_table(int pmax, std::vector<double>& out) {
    auto off = [](int j) { return (size_t)j * (j + 1) * (2 * j + 1) / 6; };
    out.assign(off(pmax + 1), 0.0);
    // quarter values d^j_{m'm}, m' >= |m| >= 0 (m >= 0 is all that the table needs)
    for (int mp = 0; mp <= pmax; ++mp)
        for (int m = 0; m <= mp; ++m) {
            long double lc = 0.0L;   // log of sqrt(C(2mp, mp+m)) 2^{-mp}
            for (int i = 1; i <= 2 * mp; ++i) lc += std::log((long double)i);
            for (int i = 1; i <= mp + m; ++i) lc -= std::log((long double)i);
            for (int i = 1; i <= mp - m; ++i) lc -= std::log((long double)i);
            long double seed = std::exp(0.5L * lc - mp * std::log(2.0L));
            if ((mp - m) & 1) seed = -seed;
            long double prev2 = 0.0L, prev1 = seed;
            for (int j = mp; j <= pmax; ++j) {
                long double v;
                if (j == mp) {
                    v = seed;
                } else if (j == 1) {
                    v = 0.0L;   // cos(pi/2) d^0_{00}
                } else {
                    long double jj = j;
                    long double c1 = jj * (2 * jj - 1) / std::sqrt((jj * jj - (long double)m * m) * (jj * jj - (long double)mp * mp));
                    long double c2 = c1 * std::sqrt(((jj - 1) * (jj - 1) - (long double)m * m) * ((jj - 1) * (jj - 1) - (long double)mp * mp)) /
                                     ((jj - 1) * (2 * jj - 1));
                    v = c1 * (-(long double)m * mp / (jj * (jj - 1))) * prev1 - c2 * prev2;
                }
                if (j > mp) {
                    prev2 = prev1;
                    prev1 = v;
                }
                // Delta_{mp, m} (b = mp, a = m) and its mirror Delta_{m, mp} = (-1)^{m - mp} Delta_{mp, m}
                out[off(j) + (size_t)m * (j + 1) + mp] = (double)v;
                out[off(j) + (size_t)mp * (j + 1) + m] = (double)(((mp - m) & 1) ? -v : v);
            }
        }
}

// g_nm = (-1)^m sqrt((n+m)!/(n-m)!) for n = 0..pmax, m = -n..n, index n(n+1)+m
void build_g_table(int pmax, std::vector<double>& g) {
    g.assign((size_t)(pmax + 1) * (pmax + 1), 1.0);
    for (int n = 0; n <= pmax; ++n)
        for (int m = -n; m <= n; ++m) {
            long double r = 1.0L;
            if (m >= 0)
                for (int i = n - m + 1; i <= n + m; ++i) r *= i;
            else
                for (int i = n + m + 1; i <= n - m; ++i) r /= i;
            double v = (double)std::sqrt(r);
            g[(size_t)n * (n + 1) + m] = (m & 1) ? -v : v;
        }
}

}  // namespace foggy
