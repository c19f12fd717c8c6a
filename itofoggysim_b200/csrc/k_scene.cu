// Scene-level kernels: Mie coefficients, plane-wave right-hand side, layout conversion between
// the reference's flat coefficient vector and the device's ragged scaled layout, and the
// cluster cross-sections.
#include "foggy_kernels.cuh"
#include "k_common.cuh"
#include "k_special.cuh"

namespace foggy {

// ---- Mie coefficients a_n, b_n (lib_mie_ss_helper_functions.f90:628-722; logarithmic
// derivative by downward recurrence 751-924; start n_c from 937-951) -----------------------
__global__ void k_mie_ab(int n_param, const double* size_param, const double* m_re, const double* m_im,
                         const int* p_of_param, int pstride, cplx* an_out, cplx* bn_out) {
    int ip = blockIdx.x * blockDim.x + threadIdx.x;
    if (ip >= n_param) return;
    double x = size_param[ip];
    cplx m = mk(m_re[ip], m_im[ip]);
    int p = p_of_param[ip];
    cplx mx = mk(m.x * x, m.y * x);
    double amx = sqrt(mx.x * mx.x + mx.y * mx.y);
    int n_c = (int)ceil(x + 4.05 * cbrt(x) + 2.0);
    int n_mx = max(n_c, (int)amx) + 15;
    cplx* an = an_out + (size_t)ip * pstride;
    cplx* bn = bn_out + (size_t)ip * pstride;
    // downward: A_{i-1} = i/(mx) - 1/(A_i + i/(mx)); keep A_n for n = 1..p in an[] temporarily
    cplx A = mk(0, 0);
    for (int i = n_mx; i >= 2; --i) {
        cplx ndm = cdiv(mk((double)i, 0), mx);
        A = ndm - cdiv(mk(1, 0), A + ndm);
        if (i - 1 <= p) an[i - 2] = A;
    }
    double jb[kMaxDegree + 2], yb[kMaxDegree + 2];
    dev_sph_jn(x, p, jb);
    dev_sph_yn(x, p, yb);
    for (int n = 1; n <= p; ++n) {
        cplx An = an[n - 1];
        double ndx = (double)n / x;
        cplx jn = mk(jb[n], 0), jnm = mk(jb[n - 1], 0), hn = mk(jb[n], yb[n]), hnm = mk(jb[n - 1], yb[n - 1]);
        cplx bufa = cdiv(An, m) + mk(ndx, 0);
        cplx bufb = m * An + mk(ndx, 0);
        an[n - 1] = cdiv(bufa * jn - jnm, bufa * hn - hnm);
        bn[n - 1] = cdiv(bufb * jn - jnm, bufb * hn - hnm);
    }
}

__global__ void k_gather_an(int n, const int* pidx, int pstride, const cplx* an_p, const cplx* bn_p,
                            cplx* an_s, cplx* bn_s) {
    int j = blockIdx.x;
    int ip = pidx[j];
    for (int t = threadIdx.x; t < pstride; t += blockDim.x) {
        an_s[(size_t)j * pstride + t] = an_p[(size_t)ip * pstride + t];
        bn_s[(size_t)j * pstride + t] = bn_p[(size_t)ip * pstride + t];
    }
}

// ---- scaled pi_nm, tau_nm of each wave (lib_math_legendre.f90:834-982; values divided by
// g_nm = (-1)^m sqrt((n+m)!/(n-m)!), which turns the recurrence into the stable normalised
// one).  Table pt[w][n(n+1)+m] (pi) and tt[...] (tau).  One thread per m >= 0. -------------
__global__ void k_pitau(int nw, const WaveDev* waves, int pmax, double* pi_out, double* tau_out) {
    int w = blockIdx.x;
    int m = threadIdx.x;
    if (m > pmax) return;
    double alpha = waves[w].alpha;
    double x = cos(alpha), s = sin(alpha);
    int S = (pmax + 1) * (pmax + 1);
    double* pi = pi_out + (size_t)w * S;
    double* tau = tau_out + (size_t)w * S;
    double sgm = (m & 1) ? -1.0 : 1.0;
    if (x == 1.0 || x == -1.0) {
        // The reference's pole table (lib_math_legendre.f90:854-920), phase removed, then
        // scaled by 1/g_{n,+-1} = -1/sqrt(n(n+1)), -sqrt(n(n+1)).  At x = -1 it sets
        // tau_n^{+-1} = -pi_n^{+-1} for odd n, which flips the sign of tau_n^{-1} there
        // relative to the limit of the general formula; kept as the reference has it.
        for (int n = max(m, 1); n <= pmax; ++n) {
            pi[n * (n + 1) + m] = 0.0;
            tau[n * (n + 1) + m] = 0.0;
            pi[n * (n + 1) - m] = 0.0;
            tau[n * (n + 1) - m] = 0.0;
        }
        if (m == 1) {
            for (int n = 1; n <= pmax; ++n) {
                double h = (double)(n * (n + 1) / 2);
                double pim = -0.5, pip = -h, taum = 0.5, taup = -h;   // with phase, x = +1
                if (x == -1.0) {
                    if (!(n & 1)) { pim = -pim; pip = -pip; }
                    else { taum = -pim; taup = -pip; }
                }
                double r = sqrt((double)n * (n + 1));
                // phase removed (odd |m|): negate; scaled by 1/g
                pi[n * (n + 1) - 1] = -pim * (-r);
                tau[n * (n + 1) - 1] = -taum * (-r);
                pi[n * (n + 1) + 1] = -pip / (-r);
                tau[n * (n + 1) + 1] = -taup / (-r);
            }
        }
        if (m == 0) { pi[0] = 0.0; tau[0] = 0.0; }
        return;
    }
    if (m == 0) {
        // tau_n^0 = -P_n^1 (no phase) -> scaled: -sqrt(n(n+1)) * Phat_n^1
        // Phat_n^1 by the normalised recurrence from Phat_1^1 = sqrt(1/2) s
        double pm2 = 0.0, pm1 = 0.0;
        for (int n = 1; n <= pmax; ++n) {
            double pn;
            if (n == 1) pn = sqrt(0.5) * s;
            else if (n == 2) pn = sqrt(3.0) * x * pm1;
            else pn = ((2.0 * n - 1.0) * x * pm1 - sqrt((n - 1.0) * (n - 1.0) - 1.0) * pm2) / sqrt((double)n * n - 1.0);
            pm2 = pm1;
            pm1 = pn;
            pi[n * (n + 1)] = 0.0;
            tau[n * (n + 1)] = -sqrt((double)n * (n + 1)) * pn;
        }
        pi[0] = 0.0;
        tau[0] = 0.0;
        return;
    }
    // Qhat_n^m = Phat_n^m / sin(alpha), Phat = sqrt((n-m)!/(n+m)!) P_n^m (no phase)
    double qmm = 1.0;
    for (int k = 1; k <= m; ++k) qmm *= sqrt((2.0 * k - 1.0) / (2.0 * k));
    for (int k = 1; k < m; ++k) qmm *= s;
    double qm2 = 0.0, qm1 = 0.0;   // Qhat_{n-2}, Qhat_{n-1}
    for (int n = m; n <= pmax; ++n) {
        double qn;
        if (n == m) qn = qmm;
        else if (n == m + 1) qn = sqrt(2.0 * m + 1.0) * x * qm1;
        else qn = ((2.0 * n - 1.0) * x * qm1 - sqrt((n - 1.0 - m) * (n - 1.0 + m)) * qm2) / sqrt((double)(n - m) * (n + m));
        double qprev = qm1;
        qm2 = qm1;
        qm1 = qn;
        double pv = m * qn;                                           // pi-hat_n^m
        double tv = n * x * qn - sqrt((double)(n + m) * (n - m)) * qprev;   // tau-hat_n^m
        pi[n * (n + 1) + m] = sgm * pv;
        tau[n * (n + 1) + m] = sgm * tv;
        // negative orders: pi_{n,-m} = -(-1)^m pi_{n,m}, tau_{n,-m} = (-1)^m tau_{n,m} (scaled)
        pi[n * (n + 1) - m] = -sgm * sgm * pv;
        tau[n * (n + 1) - m] = sgm * sgm * tv;
    }
}

// ---- right-hand side b = [a_n p ; b_n q] (lib_mie_ms_solver_interface.f90:230-315) with the
// plane-wave coefficients of lib_mie_illumination.f90:392-478 (several waves, Jones vector,
// TE swaps p and q) and :636-763 (p = tau e^{-i m beta}/(n(n+1)) e^{i(k.d + phase)}).
// One block per sphere; pq keeps the incident coefficients for the cross-sections. --------
namespace {
// p, q of one plane wave W at degree n, order m of a sphere centred at cj (pi_s, tau_s its scaled
// Legendre values there), times W.g, added to pv, qv
__device__ __forceinline__ void add_wave(const WaveDev& W, const double* cj, int m, double rn, double pi_s,
                                         double tau_s, cplx& pv, cplx& qv) {
    double d0 = cj[0] - W.d0[0], d1 = cj[1] - W.d0[1], d2 = cj[2] - W.d0[2];
    double dn = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
    double kd = W.kc[0] * d0 + W.kc[1] * d1 + W.kc[2] * d2;
    if (W.alpha == 0.0 && m != 1 && m != -1) { pi_s = 0.0; tau_s = 0.0; }
    double sb, cbv;
    sincos(-m * W.beta, &sb, &cbv);
    cplx base = mk(rn * cbv, rn * sb);
    cplx tp = mk(0, 0), tq = mk(0, 0);
    if (W.ax > 0) {
        cplx e = mk(1, 0);
        if (dn > 0.0 || W.phx != 0.0) { double ss, cc; sincos(kd + W.phx, &ss, &cc); e = mk(cc, ss); }
        tp = tp + W.ax * (e * (tau_s * base));
        tq = tq + W.ax * (e * (pi_s * base));
    }
    if (W.ay > 0) {
        cplx e = mk(1, 0);
        if (dn > 0.0 || W.phy != 0.0) { double ss, cc; sincos(kd + W.phy, &ss, &cc); e = mk(cc, ss); }
        tp = tp + W.ay * (e * (pi_s * base));    // TE: p and q swap
        tq = tq + W.ay * (e * (tau_s * base));
    }
    pv = pv + W.g * tp;
    qv = qv + W.g * tq;
}
}  // namespace

// nw waves shared by all spheres (tables [w][S]) and nl local waves per sphere (waves[j nl + l],
// tables [(j nl + l)][S]), the plane waves that stand in for Gaussian beams at each sphere
__global__ void k_rhs(SceneView sc, int nw, const WaveDev* waves, int pmax, const double* pi_tab,
                      const double* tau_tab, int nl, const WaveDev* lwaves, const double* lpi_tab,
                      const double* ltau_tab, cplx* b, cplx* pq) {
    int j = blockIdx.x;
    int pj = sc.p[j];
    int Pj = pj * (pj + 2);
    int64_t o = sc.off[j];
    int S = (pmax + 1) * (pmax + 1);
    const double* cj = sc.centres + 3 * (size_t)j;
    for (int t = threadIdx.x; t < Pj; t += blockDim.x) {
        int n = (int)sqrt((double)(t + 1));
        if ((n + 1) * (n + 1) <= t + 1) ++n;
        if (n * n > t + 1) --n;
        int m = t + 1 - n * n - n;
        cplx pv = mk(0, 0), qv = mk(0, 0);
        double rn = 1.0 / (double)(n * (n + 1));
        const int e = n * (n + 1) + m;
        for (int w = 0; w < nw; ++w)
            add_wave(waves[w], cj, m, rn, pi_tab[(size_t)w * S + e], tau_tab[(size_t)w * S + e], pv, qv);
        for (int l = 0; l < nl; ++l) {
            const size_t wl = (size_t)j * nl + l;
            add_wave(lwaves[wl], cj, m, rn, lpi_tab[wl * S + e], ltau_tab[wl * S + e], pv, qv);
        }
        pq[o + t] = pv;
        pq[o + Pj + t] = qv;
        b[o + t] = sc.an[(size_t)j * sc.pmax + n - 1] * pv;
        b[o + Pj + t] = sc.bn[(size_t)j * sc.pmax + n - 1] * qv;
    }
}

// ---- Gaussian beams in the plane-wave approximation (lib_mie_illumination.f90:781-918,
// calculation_type 3, and 1022-1050; beam functions of
// FoggySim/src/lib/field/lib_field_gaussian_beam.f90:111-891).  At each sphere the beam is replaced
// by the plane wave with the direction of its phase gradient, its phase (shifted back to the
// beam origin by 2 pi z / lambda_0) and its polarisation projected on the rotated beam axes; the
// local amplitude does not enter the coefficients (lib_mie_illumination.f90:392-478 uses only
// g, the Jones vector and the phase), and the beam's g scales them twice (:864-877). --------
namespace {
// Euler rotation, x-convention (lib_math_get_matrix_rot, lib_math_type_operator.f90:1768-1810), applied to v
__device__ void euler_apply(double phi, double theta, double psi, const double v[3], double o[3]) {
    double sph, cph, sth, cth, sps, cps;
    sincos(phi, &sph, &cph);
    sincos(theta, &sth, &cth);
    sincos(psi, &sps, &cps);
    const double a = v[0], b = v[1], c = v[2];
    o[0] = (cps * cph - cth * sph * sps) * a + (cps * sph + cth * cph * sps) * b + (sps * sth) * c;
    o[1] = (-sps * cph - cth * sph * cps) * a + (-sps * sph + cth * cph * cps) * b + (cps * sth) * c;
    o[2] = (sth * sph) * a + (-sth * cph) * b + cth * c;
}
// physicists' Hermite polynomial by its three-term recurrence
__device__ double hermite_h(int n, double x) {
    double h0 = 1.0, h1 = 2.0 * x;
    if (n == 0) return h0;
    for (int k = 1; k < n; ++k) {
        const double h2 = 2.0 * x * h1 - 2.0 * k * h0;
        h0 = h1;
        h1 = h2;
    }
    return h1;
}
}  // namespace

__global__ void k_gauss_local(SceneView sc, int nb, const GaussDev* beams, double lambda0, double n_medium,
                              WaveDev* out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= sc.n * nb) return;
    const int j = t / nb;
    const GaussDev B = beams[t - j * nb];
    const double PI_ = 3.14159265358979323846;
    const double xw[3] = {sc.centres[3 * (size_t)j] - B.d0[0], sc.centres[3 * (size_t)j + 1] - B.d0[1],
                          sc.centres[3 * (size_t)j + 2] - B.d0[2]};
    const bool rot = B.phi != 0.0 || B.theta != 0.0;
    double x[3] = {xw[0], xw[1], xw[2]};
    if (rot) euler_apply(PI_ / 2.0 + B.phi, B.theta, PI_ / 2.0 + B.phi, xw, x);
    // propagation direction: minus the phase gradient in the beam frame, normalised, rotated back
    // (get_derivative_xy / get_derivative_z, lib_field_gaussian_beam.f90:573-679)
    const double pn2 = (PI_ * n_medium) * (PI_ * n_medium), lz2 = (lambda0 * x[2]) * (lambda0 * x[2]);
    const double wx2 = B.wx0 * B.wx0, wx4 = wx2 * wx2, wy2 = B.wy0 * B.wy0, wy4 = wy2 * wy2;
    auto dxy = [&](double w4, double xy) {
        return (xy == 0.0 || x[2] == 0.0) ? 0.0 : -2.0 * PI_ * lambda0 * xy * x[2] * n_medium / (pn2 * w4 + lz2);
    };
    double dz = (2.0 * B.tem_m * wx2 + 2.0 * x[0] * x[0]) / (pn2 * wx4 + lz2);
    dz += (2.0 * B.tem_n * wy2 + 2.0 * x[1] * x[1]) / (pn2 * wy4 + lz2);
    dz += -4.0 * pn2 * x[0] * x[0] * wx4 / ((pn2 * wx4 + lz2) * (pn2 * wx4 + lz2));
    dz += -4.0 * pn2 * x[1] * x[1] * wy4 / ((pn2 * wy4 + lz2) * (pn2 * wy4 + lz2));
    dz = PI_ * n_medium * (dz * lambda0 * lambda0 / 2.0 - 2.0) / lambda0;
    double kb[3] = {-dxy(wx4, x[0]), -dxy(wy4, x[1]), -dz};
    const double kn = sqrt(kb[0] * kb[0] + kb[1] * kb[1] + kb[2] * kb[2]);
    kb[0] /= kn;
    kb[1] /= kn;
    kb[2] /= kn;
    double kv[3] = {kb[0], kb[1], kb[2]};
    if (rot) euler_apply(-PI_ / 2.0 - B.phi, -B.theta, -PI_ / 2.0 - B.phi, kb, kv);
    const double kr = sqrt(kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2]);
    const double th = (kr == 0.0) ? 0.0 : acos(kv[2] / kr);
    const double ph = (kv[0] == 0.0 && kv[1] == 0.0) ? 0.0 : atan2(kv[1], kv[0]);
    // argument of the beam at the point (get_absolute_value_and_argument, :681-799)
    const double k = 2.0 * PI_ * n_medium / lambda0, two_pi = 2.0 * PI_;
    const double zrx = PI_ * wx2 * n_medium / lambda0, zry = PI_ * wy2 * n_medium / lambda0;
    const double wx = B.wx0 * sqrt(1.0 + (x[2] / zrx) * (x[2] / zrx)), wy = B.wy0 * sqrt(1.0 + (x[2] / zry) * (x[2] / zry));
    const double crx = x[2] / (x[2] * x[2] + zrx * zrx), cry = x[2] / (x[2] * x[2] + zry * zry);
    double arg = -fmod(k * crx * x[0] * x[0] / 2.0, two_pi);
    arg = arg - fmod(k * cry * x[1] * x[1] / 2.0, two_pi);
    arg = arg - fmod(k * x[2], two_pi) + B.phase;
    arg = arg + (B.tem_m + 0.5) * atan2(x[2], zrx);
    arg = arg + (B.tem_n + 0.5) * atan2(x[2], zry);
    const double hx = hermite_h(B.tem_m, x[0] * sqrt(2.0) / wx), hy = hermite_h(B.tem_n, x[1] * sqrt(2.0) / wy);
    if (hx * hy < 0.0) arg = arg - PI_;
    arg = fmod(arg, two_pi);
    if (B.convention == 2) arg = -arg;
    if (arg < 0.0) arg = two_pi + arg;
    double phase = fmod(arg + fmod(two_pi * x[2] / lambda0, two_pi), two_pi);
    if (phase < 0.0) phase = two_pi + phase;
    // polarisation on the rotated beam axes (:329-352)
    double ax[3] = {1.0, 0.0, 0.0}, ay[3] = {0.0, 1.0, 0.0};
    if (ph != 0.0 || th != 0.0) {
        const double ex[3] = {1.0, 0.0, 0.0}, ey[3] = {0.0, 1.0, 0.0};
        euler_apply(PI_ / 2.0 + B.phi, B.theta, PI_ / 2.0 + B.phi, ex, ax);
        euler_apply(PI_ / 2.0 + B.phi, B.theta, PI_ / 2.0 + B.phi, ey, ay);
    }
    const double pxr = B.jxr * fabs(ax[0]) + B.jyr * fabs(ay[0]), pxi = B.jxi * fabs(ax[0]) + B.jyi * fabs(ay[0]);
    const double pyr = B.jyr * fabs(ay[1]) + B.jxr * fabs(ax[1]), pyi = B.jyi * fabs(ay[1]) + B.jxi * fabs(ax[1]);
    const double nrm = sqrt(pxr * pxr + pxi * pxi + pyr * pyr + pyi * pyi);
    // the plane wave as the right-hand side takes it (direction through its cartesian round trip)
    WaveDev W;
    double st_, ct_, sp_, cp_;
    sincos(th, &st_, &ct_);
    sincos(ph, &sp_, &cp_);
    W.kc[0] = k * st_ * cp_;
    W.kc[1] = k * st_ * sp_;
    W.kc[2] = k * ct_;
    const double r2 = sqrt(W.kc[0] * W.kc[0] + W.kc[1] * W.kc[1] + W.kc[2] * W.kc[2]);
    W.alpha = (r2 == 0.0) ? 0.0 : acos(W.kc[2] / r2);
    W.beta = (W.kc[0] == 0.0 && W.kc[1] == 0.0) ? 0.0 : atan2(W.kc[1], W.kc[0]);
    W.ax = hypot(pxr / nrm, pxi / nrm);
    W.phx = atan2(pxi / nrm, pxr / nrm) + phase;
    W.ay = hypot(pyr / nrm, pyi / nrm);
    W.phy = atan2(pyi / nrm, pyr / nrm) + phase;
    W.g = B.g * B.g;
    W.d0[0] = B.d0[0];
    W.d0[1] = B.d0[1];
    W.d0[2] = B.d0[2];
    out[t] = W;
}

// ---- layout conversion ---------------------------------------------------------------------
// reference flat layout (per sphere 2C entries, C = (pg+1)^2 - 1) <-> ragged scaled layout
__global__ void k_unpack(SceneView sc, int pg, const double* g, const cplx* xref, cplx* xdev) {
    int j = blockIdx.x;
    int pj = sc.p[j];
    int Pj = pj * (pj + 2);
    int C = (pg + 1) * (pg + 1) - 1;
    int64_t o = sc.off[j];
    for (int t = threadIdx.x; t < Pj; t += blockDim.x) {
        int n = (int)sqrt((double)(t + 1));
        if ((n + 1) * (n + 1) <= t + 1) ++n;
        if (n * n > t + 1) --n;
        int m = t + 1 - n * n - n;
        double rg = 1.0 / g[n * (n + 1) + m];
        xdev[o + t] = rg * xref[(size_t)2 * C * j + t];
        xdev[o + Pj + t] = rg * xref[(size_t)2 * C * j + C + t];
    }
}

// identity_ref != nullptr: entries above the sphere's own degree are copied from it (the
// identity rows of the reference operator); otherwise they are set to zero.
__global__ void k_pack(SceneView sc, int pg, const double* g, const cplx* ydev, const cplx* identity_ref,
                       cplx* yref) {
    int j = blockIdx.x;
    int pj = sc.p[j];
    int Pj = pj * (pj + 2);
    int C = (pg + 1) * (pg + 1) - 1;
    int64_t o = sc.off[j];
    for (int t = threadIdx.x; t < C; t += blockDim.x) {
        size_t ra = (size_t)2 * C * j + t, rb = ra + C;
        if (t < Pj) {
            int n = (int)sqrt((double)(t + 1));
            if ((n + 1) * (n + 1) <= t + 1) ++n;
            if (n * n > t + 1) --n;
            int m = t + 1 - n * n - n;
            double gv = g[n * (n + 1) + m];
            yref[ra] = gv * ydev[o + t];
            yref[rb] = gv * ydev[o + Pj + t];
        } else if (identity_ref) {
            yref[ra] = identity_ref[ra];
            yref[rb] = identity_ref[rb];
        } else {
            yref[ra] = mk(0, 0);
            yref[rb] = mk(0, 0);
        }
    }
}

// ---- cluster cross-sections, per sphere partial sums {ext, abs} ----------------------------
// In the scaled basis the reference weights n(n+1)(2n+1)(n-m)!/(n+m)! reduce to n(n+1)(2n+1).
__global__ void k_cross_sections(SceneView sc, const cplx* x, const cplx* pq, double* part) {
    int j = blockIdx.x;
    int pj = sc.p[j];
    int Pj = pj * (pj + 2);
    int64_t o = sc.off[j];
    double se = 0.0, sa = 0.0;
    for (int t = threadIdx.x; t < Pj; t += blockDim.x) {
        int n = (int)sqrt((double)(t + 1));
        if ((n + 1) * (n + 1) <= t + 1) ++n;
        if (n * n > t + 1) --n;
        double E = (double)(n * (n + 1) * (2 * n + 1));
        cplx a = x[o + t], bb = x[o + Pj + t];
        cplx p = pq[o + t], q = pq[o + Pj + t];
        cplx an = sc.an[(size_t)j * sc.pmax + n - 1], bn = sc.bn[(size_t)j * sc.pmax + n - 1];
        double ra = (an.x != 0.0 || an.y != 0.0) ? cdiv(mk(1, 0), an).x - 1.0 : 0.0;
        double rb = (bn.x != 0.0 || bn.y != 0.0) ? cdiv(mk(1, 0), bn).x - 1.0 : 0.0;
        se += E * ((conjg(p) * a).x + (conjg(q) * bb).x);
        sa += E * ((a.x * a.x + a.y * a.y) * ra + (bb.x * bb.x + bb.y * bb.y) * rb);
    }
    __shared__ double red[2][256];
    red[0][threadIdx.x] = se;
    red[1][threadIdx.x] = sa;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            red[0][threadIdx.x] += red[0][threadIdx.x + s];
            red[1][threadIdx.x] += red[1][threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * j] = red[0][0];
        part[2 * j + 1] = red[1][0];
    }
}

// ---- scattered field at observation points (lib_mie_ms_get_field,
// FoggySim/src/lib/mie_theory/lib_mie_multi_sphere.f90:379-434; per sphere lib_mie_ss_get_field,
// lib_mie_single_sphere.f90:1397-1582; vector spherical wave functions of
// lib_math_vector_spherical_harmonics_components_real_xu,
// libmath/src/math/lib_math_vector_spherical_harmonics.f90:132-419) -------------------------------
//   E += sum_nm E_nm i (a_nm N_nm + b_nm M_nm),  H += n_medium / c0 sum_nm E_nm (b_nm N_nm + a_nm M_nm)
//   E_nm = |E0| (2n+1) (n-m)!/(n+m)! i^n, with h_n^(1) in M, N, per sphere in its own frame,
// converted to cartesian components and summed; zero at a point inside any sphere.  One CTA per
// point, each thread a strided subset of the spheres; Legendre functions (no Condon-Shortley
// phase), pi_nm = m P_n^m / sin t and tau_nm = dP_n^m/dt by recurrence per order m.
namespace {
constexpr int kFieldThreads = 128;

// contribution of degree n and order mm to the spherical components of E and H, given P_n^mm,
// pi_n,mm, tau_n,mm and (n-mm)!/(n+mm)!
__device__ __forceinline__ void field_term(int n, int mm, double P, double pv, double tv, double ratio, cplx zn,
                                           cplx xid, double rho, cplx e, const cplx* a, const cplx* b, int base,
                                           double e0, cplx* es, cplx* hs) {
    const cplx Mt = mk(0.0, pv) * zn * e, Mp = (-tv) * (zn * e);
    const cplx Nr = ((double)(n * (n + 1)) * P / rho) * (zn * e), Nt = (tv / rho) * (xid * e),
               Np = (1.0 / rho) * (mk(0.0, pv) * (xid * e));
    const cplx Enm = ipow_mul(n, mk(e0 * (2.0 * n + 1.0) * ratio, 0.0));
    const cplx an = a[base + mm], bn = b[base + mm];
    const cplx ie = mk(-Enm.y, Enm.x);   // i E_nm
    es[0] = es[0] + ie * (an * Nr);
    es[1] = es[1] + ie * (an * Nt + bn * Mt);
    es[2] = es[2] + ie * (an * Np + bn * Mp);
    hs[0] = hs[0] + Enm * (bn * Nr);
    hs[1] = hs[1] + Enm * (bn * Nt + an * Mt);
    hs[2] = hs[2] + Enm * (bn * Np + an * Mp);
}
}  // namespace

__global__ void __launch_bounds__(kFieldThreads) k_field(SceneView sc, const double* radius_s, int pg, int C,
                                                         const cplx* x, const double* pts, double e0,
                                                         double h_factor, cplx* E_out, cplx* H_out) {
    const int ip = blockIdx.x;
    const int tid = threadIdx.x;
    __shared__ int inside;
    __shared__ double red[12][kFieldThreads];
    if (tid == 0) inside = 0;
    __syncthreads();
    const double* pt = pts + 3 * (size_t)ip;
    cplx acc[6];
    for (int c = 0; c < 6; ++c) acc[c] = mk(0.0, 0.0);
    double jb[2 * kMaxDegree + 4], yb[2 * kMaxDegree + 4];
    for (int j = tid; j < sc.n; j += kFieldThreads) {
        const double d0 = pt[0] - sc.centres[3 * (size_t)j];
        const double d1 = pt[1] - sc.centres[3 * (size_t)j + 1];
        const double d2 = pt[2] - sc.centres[3 * (size_t)j + 2];
        const double r = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
        if (!(r > radius_s[j])) {
            inside = 1;
            continue;
        }
        if (!(e0 > 1e-200)) continue;
        const double th = (r == 0.0) ? 0.0 : acos(d2 / r);
        const double ph = (d0 == 0.0 && d1 == 0.0) ? 0.0 : atan2(d1, d0);
        const double rho = sc.k * r;
        dev_sph_jn(rho, pg + 1, jb);
        dev_sph_yn(rho, pg + 1, yb);
        const double xc = cos(th), st = sin(th);
        const bool pole = (xc == 1.0 || xc == -1.0);
        const cplx* a = x + (size_t)2 * C * j;
        const cplx* b = a + C;
        cplx es[3] = {mk(0, 0), mk(0, 0), mk(0, 0)}, hs[3] = {mk(0, 0), mk(0, 0), mk(0, 0)};
        // Q_n^m = P_n^m / sin t by the LPMNS recurrence; pi_nm = m Q_n^m, tau_nm = n x Q_n^m - (n+m) Q_{n-1}^m,
        // tau_n0 = -P_n^1 = -sin t Q_n^1; negative orders from P_n^{-m} = f P_n^m, f = (-1)^m (n-m)!/(n+m)!
        // (pi_{n,-m} = -f pi_nm, tau_{n,-m} = f tau_nm); at the poles the reference's table
        // (lib_math_legendre.f90:854-920, without the phase)
        double fact2m = 1.0;   // (2m)!
        for (int m = 0; m <= pg; ++m) {
            if (m > 0) fact2m *= (2.0 * m - 1.0) * (2.0 * m);
            double sphi, cphi;
            sincos((double)m * ph, &sphi, &cphi);
            const cplx ep = mk(cphi, sphi), em = mk(cphi, -sphi);
            const int mq = m == 0 ? 1 : m;   // order of the Q sequence (Q^1 for tau_n0)
            double qmm = 1.0;
            for (int q = 1; q <= mq; ++q) qmm *= (2.0 * q - 1.0);
            for (int q = 1; q < mq; ++q) qmm *= st;
            double qc = qmm, qprev = 0.0;                       // Q_n^mq at n = mq, and n - 1
            double pc = m == 0 ? 1.0 : qmm * st, pprev = 0.0;   // P_n^m at n = m, and n - 1
            double fr = 1.0 / fact2m;                           // (n-m)!/(n+m)! at n = m
            int nq = mq, np_ = m;
            for (int n = max(m, 1); n <= pg; ++n) {
                while (np_ < n) {   // advance P_n^m and (n-m)!/(n+m)!
                    ++np_;
                    const double pn = ((2.0 * np_ - 1.0) * xc * pc - (np_ + m - 1.0) * pprev) / (np_ - m);
                    pprev = pc;
                    pc = pn;
                    fr *= (double)(np_ - m) / (double)(np_ + m);
                }
                while (nq < n) {    // advance Q_n^mq
                    ++nq;
                    const double qn = ((2.0 * nq - 1.0) * xc * qc - (nq + mq - 1.0) * qprev) / (nq - mq);
                    qprev = qc;
                    qc = qn;
                }
                const cplx zn = mk(jb[n], yb[n]);
                const cplx zm1 = mk(jb[n - 1], yb[n - 1]), zp1 = mk(jb[n + 1], yb[n + 1]);
                const cplx xid = 0.5 * (rho * zm1 + zn - rho * zp1);
                const int base = n * n - 1 + n;
                if (m == 0) {
                    const double P0 = pole ? ((xc < 0.0 && (n & 1)) ? -1.0 : 1.0) : pc;
                    const double t0 = pole ? 0.0 : -st * qc;
                    field_term(n, 0, P0, 0.0, t0, 1.0, zn, xid, rho, ep, a, b, base, e0, es, hs);
                    continue;
                }
                double pip, taup, pim, taum, Pp, Pm;
                if (pole) {
                    Pp = Pm = 0.0;
                    pip = taup = pim = taum = 0.0;
                    if (m == 1) {
                        const double N2 = (double)(n * (n + 1) / 2);
                        if (xc > 0.0) {
                            pip = N2; pim = 0.5; taup = N2; taum = -0.5;
                        } else if ((n & 1) == 0) {
                            pip = -N2; pim = -0.5; taup = N2; taum = -0.5;
                        } else {
                            pip = N2; pim = 0.5; taup = -N2; taum = -0.5;
                        }
                    }
                } else {
                    const double f = (m & 1) ? -fr : fr;
                    Pp = pc;
                    Pm = f * pc;
                    pip = m * qc;
                    taup = n * xc * qc - (n + m) * qprev;
                    pim = -f * pip;
                    taum = f * taup;
                }
                field_term(n, m, Pp, pip, taup, fr, zn, xid, rho, ep, a, b, base, e0, es, hs);
                field_term(n, -m, Pm, pim, taum, 1.0 / fr, zn, xid, rho, em, a, b, base, e0, es, hs);
            }
        }
        const double ct = xc, cp = cos(ph), sp = sin(ph);
        const cplx ex = st * cp * es[0] + ct * cp * es[1] - sp * es[2];
        const cplx ey = st * sp * es[0] + ct * sp * es[1] + cp * es[2];
        const cplx ez = ct * es[0] - st * es[1];
        const cplx hx = st * cp * hs[0] + ct * cp * hs[1] - sp * hs[2];
        const cplx hy = st * sp * hs[0] + ct * sp * hs[1] + cp * hs[2];
        const cplx hz = ct * hs[0] - st * hs[1];
        acc[0] = acc[0] + ex;
        acc[1] = acc[1] + ey;
        acc[2] = acc[2] + ez;
        acc[3] = acc[3] + h_factor * hx;
        acc[4] = acc[4] + h_factor * hy;
        acc[5] = acc[5] + h_factor * hz;
    }
    for (int c = 0; c < 6; ++c) {
        red[2 * c][tid] = acc[c].x;
        red[2 * c + 1][tid] = acc[c].y;
    }
    __syncthreads();
    for (int s_ = kFieldThreads / 2; s_ > 0; s_ >>= 1) {
        if (tid < s_)
            for (int c = 0; c < 12; ++c) red[c][tid] += red[c][tid + s_];
        __syncthreads();
    }
    if (tid < 6) {
        const cplx v = inside ? mk(0.0, 0.0) : mk(red[2 * tid][0], red[2 * tid + 1][0]);
        if (tid < 3) E_out[3 * (size_t)ip + tid] = v;
        else H_out[3 * (size_t)ip + tid - 3] = v;
    }
}

}  // namespace foggy
