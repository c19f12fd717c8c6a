// Translation coefficients A, B of one sphere pair in the scaled basis, for the parity entry
// point foggy_translation_coefficients (the reference's
// lib_math_vector_spherical_harmonics_translation_coeff_r,
// libmath/src/math/lib_math_vector_spherical_harmonics.f90:1354-1585).  One CTA builds the
// Wigner small-d table of the pair's polar angle by the Jacobi recurrence, the axial
// coefficients from the 3j tables (gaunt.cpp) and z_p(kd), and forms
//
//   A(theta, phi)_{nm, nu mu} = e^{i(mu-m)phi} sum_k d^n_{mk}(theta) d^nu_{mu k}(theta) A_ax(k; n, nu)
//
// (and B alike) entry by entry.
#include "k_common.cuh"
#include "k_special.cuh"

namespace foggy {

namespace {
constexpr int kThreads = 256;
constexpr int kTab = 1024;

// one (m', m) column index c < (pp+1)^2 -> (m', m)
__device__ __forceinline__ void decode_col(int c, int& mp, int& m) {
    int q = (int)__fsqrt_rn((float)c);
    if ((q + 1) * (q + 1) <= c) ++q;
    if (q * q > c) --q;
    mp = q;
    m = c - q * q - q;
}

__host__ __device__ inline size_t align2(size_t v) { return (v + 1) & ~(size_t)1; }

struct Smem {
    double* dq;    // quarter Wigner-d table, degrees <= pp
    double* jb;    // j_p(rho)
    double* yb;    // y_p(rho)
    cplx* zeta;    // i^p z_p(rho)
    cplx* eph;     // e^{i mu phi}, |mu| <= pp
    cplx* x1;      // phase-multiplied source (a | b), then the axially translated field (a | b)
    cplx* xr;      // rotated source (a | b)
    cplx* tab;     // axial coefficients of one k-chunk: (A, B) pairs
    cplx* acc;     // target accumulator (a | b)
    double* geom;  // rho, theta, phi
};

__host__ __device__ inline size_t smem_doubles(int pp) {
    size_t P = (size_t)pp * (pp + 2);
    return align2(dq_size(pp)) + 2 * align2(2 * pp + 3) + 2 * (2 * pp + 3) + 2 * (2 * pp + 1) + 3 * 2 * (2 * P) +
           2 * 2 * kTab + 4;
}

__device__ inline Smem carve(double* base, int pp) {
    Smem s;
    size_t o = 0;
    int P = pp * (pp + 2);
    s.dq = base + o;   o += align2(dq_size(pp));
    s.jb = base + o;   o += align2(2 * pp + 3);
    s.yb = base + o;   o += align2(2 * pp + 3);
    s.zeta = reinterpret_cast<cplx*>(base + o); o += 2 * (2 * pp + 3);
    s.eph = reinterpret_cast<cplx*>(base + o);  o += 2 * (2 * pp + 1);
    s.x1 = reinterpret_cast<cplx*>(base + o);   o += 2 * (2 * P);
    s.xr = reinterpret_cast<cplx*>(base + o);   o += 2 * (2 * P);
    s.acc = reinterpret_cast<cplx*>(base + o);  o += 2 * (2 * P);
    s.tab = reinterpret_cast<cplx*>(base + o);  o += 2 * 2 * kTab;
    s.geom = base + o;
    return s;
}

// Column (m', m), m' >= |m|, of the quarter d-table for j = m'..jmax by the upward three-term
// recurrence of the Jacobi polynomials behind d^j_{m'm}; division-free with the tables
//   rs[j][m] = sqrt(j^2 - m^2), irs[j][m] = 1/sqrt(j^2 - m^2), rj[j] = {1/(j(j-1)), 1/((j-1)(2j-1))}.
__device__ inline void dq_column2(double* dq, int mp, int m, int jmax, double cb, double ch, double sh,
                                  const DTabs& t) {
    int J = mp;
    int am = m < 0 ? -m : m;
    double v = sgn(J - m) * t.sqrt_binom[J * (2 * t.K + 1) + (m + t.K)] * ipow_d(ch, J + m) * ipow_d(sh, J - m);
    dq[dq_index(J, mp, m)] = v;
    double prev2 = 0.0, prev1 = v;
    const int W = t.K + 1;
    double mmp = (double)(m * mp);
    for (int j = J + 1; j <= jmax; ++j) {
        double val;
        if (j == 1) {
            val = cb * prev1;
        } else {
            double jj = (double)j;
            double c1 = jj * (2.0 * jj - 1.0) * t.irs[j * W + am] * t.irs[j * W + mp];
            double c2 = c1 * t.rs[(j - 1) * W + am] * t.rs[(j - 1) * W + mp] * t.rj[2 * j + 1];
            val = c1 * (cb - mmp * t.rj[2 * j]) * prev1 - c2 * prev2;
        }
        dq[dq_index(j, mp, m)] = val;
        prev2 = prev1;
        prev1 = val;
    }
}

// The reference evaluates its Legendre functions at x = cos(theta) with sqrt(|1 - x^2|) as
// the sine (LPMNS, lib_math_legendre.f90:68-126); the half angles are taken from that same
// (x, s) so that the rotation sees the angle the reference sees, also where cos(theta) rounds
// to +-1.
__device__ __forceinline__ void half_angles(double theta, double& cb, double& cb2, double& sb2) {
    cb = cos(theta);
    double sbf = sqrt(fabs(1.0 - cb * cb));
    if (cb >= 0.0) {
        cb2 = sqrt(0.5 * (1.0 + cb));
        sb2 = 0.5 * sbf / cb2;
    } else {
        sb2 = sqrt(0.5 * (1.0 - cb));
        cb2 = 0.5 * sbf / sb2;
    }
}

// A_ax(k; n, nu), B_ax(k; n, nu) for k >= 0 from the 3j tables and zeta
__device__ __forceinline__ void axial_coeff(const AxialView& ax, const cplx* zeta, int k, int n, int nu, cplx& A,
                                            cplx& B) {
    int S = ax.pmax + 1;
    int o = ax.offset[((size_t)k * S + n) * S + nu];
    int qm = min(n, nu);
    const double* ga = ax.ga + o;
    const double* gb = ax.gb + o;
    int p = n + nu;
    double g1 = __ldg(ga);
    double ax_ = g1 * zeta[p].x, ay_ = g1 * zeta[p].y, bx_ = 0, by_ = 0;
    for (int q = 1; q <= qm; ++q) {
        p -= 2;
        double g1q = __ldg(ga + q);
        double g2q = __ldg(gb + q);
        cplx z0 = zeta[p], z1 = zeta[p + 1];
        ax_ += g1q * z0.x;
        ay_ += g1q * z0.y;
        bx_ += g2q * z1.x;
        by_ += g2q * z1.y;
    }
    A = mk(ax_, ay_);
    B = mk(bx_, by_);
}

}  // namespace

size_t translation_pair_smem_bytes(int pmax) { return smem_doubles(pmax) * sizeof(double); }

// A, B of one translation in the scaled basis, row (n, m) major: rows n = 1..pn, columns
// nu = 1..pnu; one CTA.
__global__ void __launch_bounds__(kThreads) k_translation_pair(AxialView ax, DTabs dt, double x, double theta,
                                                               double phi, int pn, int pnu, int z, cplx* A,
                                                               cplx* B) {
    extern __shared__ double smem_t[];
    const int pp = max(pn, pnu);
    Smem s = carve(smem_t, pp);
    int tid = threadIdx.x;
    const int P = pn + pnu + 1;
    if (tid == 0) dev_sph_jn(x, P, s.jb);
    if (tid == 1 && z != 1) dev_sph_yn(x, P, s.yb);
    for (int t = tid; t < 2 * pp + 1; t += blockDim.x) {
        double sn, cs;
        sincos((double)(t - pp) * phi, &sn, &cs);
        s.eph[t] = mk(cs, sn);
    }
    double cb, cb2, sb2;
    half_angles(theta, cb, cb2, sb2);
    for (int cc = tid; cc < (pp + 1) * (pp + 1); cc += blockDim.x) {
        int mp, m;
        decode_col(cc, mp, m);
        dq_column2(s.dq, mp, m, pp, cb, cb2, sb2, dt);
    }
    __syncthreads();
    for (int p = tid; p <= P; p += blockDim.x) s.zeta[p] = zeta_of(z, p, s.jb, s.yb);
    __syncthreads();
    int Pn = pn * (pn + 2), Pnu = pnu * (pnu + 2);
    for (int t = tid; t < Pn * Pnu; t += blockDim.x) {
        int r = t / Pnu, cidx = t % Pnu;
        int n, m, nu, mu;
        decode_nm(r, n, m);
        decode_nm(cidx, nu, mu);
        cplx sa = mk(0, 0), sb = mk(0, 0);
        int kk = min(n, nu);
        for (int k = -kk; k <= kk; ++k) {
            cplx Aa, Bb;
            axial_coeff(ax, s.zeta, k < 0 ? -k : k, n, nu, Aa, Bb);
            if (k < 0) Bb = mk(-Bb.x, -Bb.y);
            double f = dq_get(s.dq, n, m, k) * dq_get(s.dq, nu, mu, k);
            sa = sa + f * Aa;
            sb = sb + f * Bb;
        }
        cplx e = s.eph[mu + pp] * conjg(s.eph[m + pp]);
        A[t] = e * sa;
        B[t] = e * sb;
    }
}

}  // namespace foggy
