// Direct sphere-sphere coupling operator (the reference's
// lib_mie_ms_solver_calculate_vector_b_without_transposed_all,
// FoggySim/src/lib/mie_theory/lib_mie_ms_solver_interface.f90:806-998):
//
//   y_j = x_j + diag(a_n, b_n) sum_{l != j} [A x_a + B x_b ; B x_a + A x_b](k (d_l - d_j))
//
// The reference builds the full O(p^4) translation matrices A, B from Wigner-3j sums for every
// pair and every matvec (lib_math_vector_spherical_harmonics.f90:1354-1585).  Here each pair
// applies the same operator in O(p^3) as rotate -> axial translate -> rotate back, in the basis
// x_nm / g_nm (g_nm = (-1)^m sqrt((n+m)!/(n-m)!)), where
//
//   A(theta, phi)_{nm, nu mu} = e^{i(mu-m)phi} sum_k d^n_{mk}(theta) d^nu_{mu k}(theta) A_ax(k; n, nu)
//
// exactly (rotations do not mix degrees).  A_ax/B_ax come from the precomputed 3j tables
// (gaunt.cpp) and z_p(kd); the Wigner small-d table is built per pair in shared memory.
//
// The a and b parts stay separate throughout: combining them as a +- b would diagonalise the
// axial block but loses the relative precision of the smaller part when |A| >> |B| (large
// Hankel values at small kd), which the FP64 parity with the reference does not allow.
//
// Work decomposition.  Spheres are grouped into buckets of similar truncation order; one launch
// per (target bucket, source bucket) sizes its shared memory for the larger order of the two.
// One CTA owns one target sphere and a strided subset of one source bucket.  Per source pair:
//   1. geometry; warp 0 runs the Bessel recurrences and the phases, the other warps build the
//      d-table columns; every thread prefetches its part of the source vector;
//   2. the source with the phase e^{i mu phi}; zeta_p = i^p z_p;
//   3. rotation, one thread per (degree, |k|, a|b);
//   4. axial step in chunks of k: the coefficients A, B of the chunk are built in parallel
//      over (k, n, nu) into shared memory, then applied, one thread per (n, |k|, a|b);
//   5. rotation back into the target accumulator, one thread per (n, |m|, a|b).
// The CTA's partial sum goes to its own slab that k_direct_finish adds in a fixed order, so
// results are bit-reproducible.
#include "foggy_kernels.cuh"
#include "k_special.cuh"

#include <cstdlib>

namespace foggy {

namespace {
constexpr int kThreads = 256;
constexpr int kTab = 1024;       // axial coefficient pairs per chunk (A+B, A-B)
constexpr int kMaxPrefetch = 4;  // source entries a thread keeps in registers

__device__ __forceinline__ cplx ipow_mul(int p, cplx c) {
    switch (p & 3) {
        case 0: return c;
        case 1: return mk(-c.y, c.x);
        case 2: return mk(-c.x, -c.y);
        default: return mk(c.y, -c.x);
    }
}
__device__ __forceinline__ void decode_nm(int t, int& n, int& m) {
    int nn = (int)__fsqrt_rn((float)(t + 1));
    if ((nn + 1) * (nn + 1) <= t + 1) ++nn;
    if (nn * nn > t + 1) --nn;
    n = nn;
    m = t + 1 - nn * nn - nn;
}
// u = 0.. over (n >= 1, 0 <= k <= n) in order
__device__ __forceinline__ void decode_nk(int u, int& n, int& k) {
    int nn = (int)((-1.0f + __fsqrt_rn(9.0f + 8.0f * (float)u)) * 0.5f);
    if (nn < 1) nn = 1;
    while (nn > 1 && (nn - 1) * (nn + 2) / 2 > u) --nn;
    while (nn * (nn + 3) / 2 <= u) ++nn;
    n = nn;
    k = u - (nn - 1) * (nn + 2) / 2;
}
__device__ __forceinline__ double sgn(int e) { return (e & 1) ? -1.0 : 1.0; }
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

// entry d^j_{mu k} of a full matrix from the quarter table, k >= 0, without branches:
//   |mu| <= k : (-1)^{k-mu} dq(k, mu);  mu > k : dq(mu, k);  mu < -k : (-1)^{k-mu} dq(-mu, -k)
__device__ __forceinline__ double d_col(const double* dq, int db, int mu, int k) {
    int amu = mu < 0 ? -mu : mu;
    int mp = max(k, amu);
    int m = (amu <= k) ? mu : (mu > 0 ? k : -k);
    double s = (mu > k) ? 1.0 : sgn(k - mu);
    return s * dq[db + mp * (mp + 1) + m];
}
// entry d^n_{m k} of a full matrix from the quarter table, m >= 0:
//   |k| <= m : dq(m, k);  k > m : (-1)^{k-m} dq(k, m);  k < -m : dq(-k, -m)
__device__ __forceinline__ double d_row(const double* dq, int db, int m, int k) {
    int ak = k < 0 ? -k : k;
    int mp = max(m, ak);
    int mm = (ak <= m) ? k : (k > 0 ? m : -m);
    double s = (k > m) ? sgn(k - m) : 1.0;
    return s * dq[db + mp * (mp + 1) + mm];
}

}  // namespace

// ---------------------------------------------------------------------------------------------
// Scalar coaxial coefficients of the unordered pairs (geometry only; once per scene).
__global__ void k_pair_sizes(SceneView sc, int64_t* sizes) {
    int s = blockIdx.x;
    int ps = sc.p[s];
    for (int t = s + 1 + threadIdx.x; t < sc.n; t += blockDim.x)
        sizes[pair_index(s, t, sc.n)] = pair_block_size(ps, sc.p[t]);
}

// One CTA per (sphere s, chunk c) walks t = s + 1 + c, s + 1 + c + chunks, ...:
//   S(k; a, b) = sum_q (2p+1)(a b p; -k k 0)(a b p; 0 0 0) i^p z_p(k |d_t - d_s|),  p = a + b - 2q
__global__ void __launch_bounds__(kThreads) k_pair_s(SceneView sc, SGaunt g, int z, const int64_t* pair_off,
                                                     cplx* stab, int chunks) {
    __shared__ double jb[2 * kMaxDegree + 8], yb[2 * kMaxDegree + 8];
    __shared__ cplx zeta[2 * kMaxDegree + 8];
    __shared__ double rho_s;
    const int s = blockIdx.x;
    const int ps = sc.p[s];
    const double* cs = sc.centres + 3 * (size_t)s;
    for (int t = s + 1 + blockIdx.y; t < sc.n; t += chunks) {
        const int pt = sc.p[t];
        const int P = ps + pt + 2;
        if (threadIdx.x == 0) {
            const double* ct = sc.centres + 3 * (size_t)t;
            double d0 = sc.k * (ct[0] - cs[0]);
            double d1 = sc.k * (ct[1] - cs[1]);
            double d2 = sc.k * (ct[2] - cs[2]);
            rho_s = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
        }
        __syncthreads();
        if (threadIdx.x == 0) dev_sph_jn(rho_s, P, jb);
        if (threadIdx.x == 32 && z != 1) dev_sph_yn(rho_s, P, yb);
        __syncthreads();
        for (int p = threadIdx.x; p <= P; p += blockDim.x) zeta[p] = zeta_of(z, p, jb, yb);
        __syncthreads();
        cplx* out = stab + pair_off[pair_index(s, t, sc.n)];
        const int km = min(ps, pt);
        const int64_t tot = pair_block_size(ps, pt);
        for (int64_t e = threadIdx.x; e < tot; e += blockDim.x) {
            // block k: (ps + 2 - k) x (pt + 2 - k)
            int k = 0;
            while (k < km && pair_block_offset(k + 1, ps + 2, pt + 2) <= e) ++k;
            int64_t r = e - pair_block_offset(k, ps + 2, pt + 2);
            int cols = pt + 2 - k;
            int aa = k + (int)(r / cols), bb = k + (int)(r % cols);
            const int W = g.NM - k + 1;
            const size_t plane = (size_t)W * W;
            const double* gp = g.gs + g.koff[k] + (size_t)(aa - k) * W + (bb - k);
            int qm = min(aa, bb);
            int p = aa + bb;
            double sx = 0.0, sy = 0.0;
            for (int q = 0; q <= qm; ++q, p -= 2) {
                double c = __ldg(gp + q * plane);
                sx += c * zeta[p].x;
                sy += c * zeta[p].y;
            }
            out[e] = mk(sx, sy);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads, 3) k_direct(DirectArgs a, DirectBucket bk) {
    extern __shared__ double smem_d[];
    const SceneView& sc = a.sc;
    const int pp = bk.pp;
    Smem s = carve(smem_d, pp);
    const int j = bk.targets[blockIdx.x];
    const int c = blockIdx.y;
    if (!sc.couple[j]) return;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nthr = blockDim.x;
    const int pj = sc.p[j];
    const int Pj = pj * (pj + 2);
    for (int t = tid; t < 2 * Pj; t += nthr) s.acc[t] = mk(0, 0);
    const double* cj = sc.centres + 3 * (size_t)j;

    for (int i = c; i < bk.nsources; i += bk.chunks) {
        const int l = bk.sources[i];
        if (l == j) continue;
        const int pl = sc.p[l];
        const int Pl = pl * (pl + 2);
        const int pq = max(pj, pl);
        const int P = pj + pl + 1;
        // ---- 1. geometry, then tables; source entries prefetched into registers --------------
        if (tid == 0) {
            const double* cl = sc.centres + 3 * (size_t)l;
            double d0 = sc.k * (cl[0] - cj[0]);
            double d1 = sc.k * (cl[1] - cj[1]);
            double d2 = sc.k * (cl[2] - cj[2]);
            double r = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
            s.geom[0] = r;
            s.geom[1] = (r == 0.0) ? 0.0 : acos(d2 / r);
            s.geom[2] = (d0 == 0.0 && d1 == 0.0) ? 0.0 : atan2(d1, d0);
        }
        cplx pa[kMaxPrefetch], pb[kMaxPrefetch];
        const cplx* xl = a.x + sc.off[l];
#pragma unroll
        for (int q = 0; q < kMaxPrefetch; ++q) {
            int t = tid + q * nthr;
            if (t < Pl) {
                pa[q] = xl[t];
                pb[q] = xl[Pl + t];
            }
        }
        __syncthreads();
        if (warp == 0) {
            double rho = s.geom[0], phi = s.geom[2];
            if (!a.pt.stab) {
                if (lane == 0) dev_sph_jn(rho, P, s.jb);
                else if (lane == 1 && a.z != 1) dev_sph_yn(rho, P, s.yb);
            }
            for (int mu = -pq + lane; mu <= pq; mu += 32) {
                double sn, cs;
                sincos((double)mu * phi, &sn, &cs);
                s.eph[mu + pp] = mk(cs, sn);
            }
        } else {
            double cb, cb2, sb2;
            half_angles(s.geom[1], cb, cb2, sb2);
            int ncol = (pq + 1) * (pq + 1);
            for (int cc = tid - 32; cc < ncol; cc += nthr - 32) {
                int mp, m;
                decode_col(cc, mp, m);
                dq_column2(s.dq, mp, m, pq, cb, cb2, sb2, a.dt);
            }
        }
        __syncthreads();
        // ---- 2. x1 = e^{i mu phi} x (a | b); zeta ---------------------------------------------
#pragma unroll
        for (int q = 0; q < kMaxPrefetch; ++q) {
            int t = tid + q * nthr;
            if (t < Pl) {
                int nu, mu;
                decode_nm(t, nu, mu);
                cplx e = s.eph[mu + pp];
                s.x1[t] = e * pa[q];
                s.x1[Pl + t] = e * pb[q];
            }
        }
        for (int t = kMaxPrefetch * nthr + tid; t < Pl; t += nthr) {   // orders above the prefetch
            int nu, mu;
            decode_nm(t, nu, mu);
            cplx e = s.eph[mu + pp];
            s.x1[t] = e * xl[t];
            s.x1[Pl + t] = e * xl[Pl + t];
        }
        if (!a.pt.stab)
            for (int p = tid; p <= P; p += nthr) s.zeta[p] = zeta_of(a.z, p, s.jb, s.yb);
        __syncthreads();
        // ---- 3. rotate the source: x'_nu[+-k] = sum_mu d^nu_{mu k} x1_nu[mu] (and partner) ----
        {
            int items = pl * (pl + 3);   // (nu, k >= 0) x {a, b}
            for (int t = tid; t < items; t += nthr) {
                int part = t & 1;
                int nu, k;
                decode_nk(t >> 1, nu, k);
                int base = nu * nu - 1 + nu;
                int db = dq_base(nu);
                const cplx* xv = s.x1 + part * Pl + base;
                double px = 0, py = 0, mx = 0, my = 0;
                for (int mu = -nu; mu <= nu; ++mu) {
                    double d = d_col(s.dq, db, mu, k);
                    double dm = sgn(k - mu) * d;
                    cplx x1p = xv[mu], x1m = xv[-mu];
                    px += d * x1p.x;
                    py += d * x1p.y;
                    mx += dm * x1m.x;
                    my += dm * x1m.y;
                }
                cplx* out = s.xr + part * Pl + base;
                out[k] = mk(px, py);
                if (k > 0) out[-k] = mk(mx, my);
            }
        }
        __syncthreads();
        // ---- 4. axial step in chunks of k -----------------------------------------------------
        {
            const int kmax = min(pj, pl);
            // orders |k| > pl of the target receive nothing from this source
            if (pj > kmax) {
                int items = Pj;
                for (int t = tid; t < 2 * items; t += nthr) {
                    int part = t >= items;
                    int n, k;
                    decode_nm(t - part * items, n, k);
                    if (k > kmax || k < -kmax) s.x1[part * Pj + t - part * items] = mk(0, 0);
                }
            }
            int k0 = 0;
            while (k0 <= kmax) {
                // chunk [k0, k1): entries (k, n, nu) with n, nu >= max(1, k)
                int k1 = k0, tot = 0;
                while (k1 <= kmax) {
                    int lo = max(1, k1);
                    int e = (pj - lo + 1) * (pl - lo + 1);
                    if (tot + e > kTab && k1 > k0) break;
                    tot += e;
                    ++k1;
                }
                // build (A, B) of the chunk
                for (int t = tid; t < tot; t += nthr) {
                    int k = k0, off = 0;
                    for (;;) {
                        int lo = max(1, k);
                        int e = (pj - lo + 1) * (pl - lo + 1);
                        if (t < off + e) break;
                        off += e;
                        ++k;
                    }
                    int lo = max(1, k);
                    int r = t - off;
                    int nnu = pl - lo + 1;
                    int n = lo + r / nnu, nu = lo + r % nnu;
                    if (a.pt.stab) {
                        // A, B from the pair's scalar coaxial coefficients S(k; n, nu - 1 .. nu + 1)
                        const bool jfirst = j < l;
                        const int s_ = jfirst ? j : l, t_ = jfirst ? l : j;
                        const int ps = jfirst ? pj : pl, pt = jfirst ? pl : pj;
                        const cplx* blk = a.pt.stab + a.pt.pair_off[pair_index(s_, t_, sc.n)] +
                                          pair_block_offset(k, ps + 2, pt + 2);
                        const int cols = pt + 2 - k;
                        auto T = [&](int dn, int dnu) {
                            int ia = jfirst ? dn : dnu, ib = jfirst ? dnu : dn;
                            return blk[(ia - k) * cols + (ib - k)];
                        };
                        cplx S0 = T(n, nu), Sp = T(n, nu + 1);
                        cplx Sm = (nu - 1 >= k) ? T(n, nu - 1) : mk(0, 0);
                        const int W = a.dt.K + 1;
                        const double x = s.geom[0];
                        double pre = sgn(k) * (2.0 * nu + 1.0) / (2.0 * n * (n + 1.0));
                        double c0 = 2.0 * nu * (nu + 1.0);
                        double c1 = x * 2.0 * nu * a.dt.rs[(nu + 1) * W + k] / (2.0 * nu + 1.0);
                        double c2 = x * 2.0 * (nu + 1.0) * a.dt.rs[nu * W + k] / (2.0 * nu + 1.0);
                        // A = pre [c0 S0 + i (c1 Sp - c2 Sm)],  B = pre 2 i k x S0
                        cplx d = c1 * Sp - c2 * Sm;
                        s.tab[2 * t] = pre * mk(c0 * S0.x - d.y, c0 * S0.y + d.x);
                        double bk2 = pre * 2.0 * k * x;
                        s.tab[2 * t + 1] = mk(-bk2 * S0.y, bk2 * S0.x);
                        continue;
                    }
                    // q-major 3j table: neighbouring threads read neighbouring (n, nu)
                    const int W = a.ax.pmax - lo + 1;
                    const size_t plane = (size_t)W * W;
                    const double2* g = a.ax.gab + a.ax.koff[k] + (size_t)(n - lo) * W + (nu - lo);
                    int qm = min(n, nu);
                    int p = n + nu;
                    double2 g0 = __ldg(g);
                    double ax_ = g0.x * s.zeta[p].x, ay_ = g0.x * s.zeta[p].y, bx_ = 0.0, by_ = 0.0;
                    for (int q = 1; q <= qm; ++q) {
                        p -= 2;
                        double2 gq = __ldg(g + q * plane);
                        cplx z0 = s.zeta[p], z1 = s.zeta[p + 1];
                        ax_ += gq.x * z0.x;
                        ay_ += gq.x * z0.y;
                        bx_ += gq.y * z1.x;
                        by_ += gq.y * z1.y;
                    }
                    s.tab[2 * t] = mk(ax_, ay_);
                    s.tab[2 * t + 1] = mk(bx_, by_);
                }
                __syncthreads();
                // apply: items (n, k >= 0) x {a, b}
                int items = 0;
                for (int k = k0; k < k1; ++k) items += pj - max(1, k) + 1;
                for (int t = tid; t < 2 * items; t += nthr) {
                    int part = t & 1;
                    int w = t >> 1;
                    int k = k0, off = 0, toff = 0;
                    for (;;) {
                        int lo = max(1, k);
                        int e = pj - lo + 1;
                        if (w < off + e) break;
                        off += e;
                        toff += e * (pl - lo + 1);
                        ++k;
                    }
                    int lo = max(1, k);
                    int n = lo + (w - off);
                    int nnu = pl - lo + 1;
                    const cplx* row = s.tab + 2 * (toff + (n - lo) * nnu);
                    // a' = A a + B b, b' = B a + A b at +k;  a' = A a - B b, b' = -B a + A b at -k
                    const cplx* xs = s.xr + part * Pl;          // same part
                    const cplx* xo = s.xr + (1 - part) * Pl;    // other part
                    cplx yp = mk(0, 0), ym = mk(0, 0);
                    for (int nu = lo; nu <= pl; ++nu) {
                        cplx A = row[2 * (nu - lo)], B = row[2 * (nu - lo) + 1];
                        int base = nu * nu - 1 + nu;
                        yp = yp + A * xs[base + k] + B * xo[base + k];
                        if (k > 0) ym = ym + A * xs[base - k] - B * xo[base - k];
                    }
                    int ob = part * Pj + n * n - 1 + n;
                    s.x1[ob + k] = yp;
                    if (k > 0) s.x1[ob - k] = ym;
                }
                __syncthreads();
                k0 = k1;
            }
        }
        // ---- 5. rotate back into the accumulator ------------------------------------------------
        {
            int items = pj * (pj + 3);   // (n, m >= 0) x {a, b}
            for (int t = tid; t < items; t += nthr) {
                int part = t & 1;
                int n, m;
                decode_nk(t >> 1, n, m);
                int base = n * n - 1 + n;
                int db = dq_base(n);
                const cplx* yv = s.x1 + part * Pj + base;
                double px = 0, py = 0, mx = 0, my = 0;
                for (int k = -n; k <= n; ++k) {
                    double d = d_row(s.dq, db, m, k);
                    double dm = sgn(m - k) * d;
                    cplx yp = yv[k], ym = yv[-k];
                    px += d * yp.x;
                    py += d * yp.y;
                    mx += dm * ym.x;
                    my += dm * ym.y;
                }
                cplx* acc = s.acc + part * Pj + base;
                cplx e = s.eph[m + pp];
                acc[m] = acc[m] + conjg(e) * mk(px, py);
                if (m > 0) acc[-m] = acc[-m] + e * mk(mx, my);
            }
        }
        __syncthreads();
    }
    cplx* out = a.partial + (size_t)(bk.slab + c) * a.n_unk + sc.off[j];
    for (int t = tid; t < 2 * Pj; t += nthr) out[t] = s.acc[t];
    // slabs of this source bucket that launches with fewer chunks leave unused
    if (c == bk.chunks - 1)
        for (int e = c + 1; e < a.cmax; ++e) {
            cplx* z = a.partial + (size_t)(bk.slab + e) * a.n_unk + sc.off[j];
            for (int t = tid; t < 2 * Pj; t += nthr) z[t] = mk(0, 0);
        }
}

size_t direct_smem_bytes(int pp) { return smem_doubles(pp) * sizeof(double); }

void launch_direct(const DirectArgs& a, const DirectBucket& b, cudaStream_t s) {
    size_t smem = direct_smem_bytes(b.pp);
    dim3 grid(b.ntargets, b.chunks);
    cudaFuncSetAttribute(k_direct, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_direct<<<grid, kThreads, smem, s>>>(a, b);
}

// y = x + T (sum of the slabs) for coupled spheres, y = x otherwise
__global__ void k_direct_finish(SceneView sc, const cplx* x, const cplx* partial, int slabs, int64_t n_unk,
                                cplx* y) {
    int j = blockIdx.x;
    int pj = sc.p[j];
    int Pj = pj * (pj + 2);
    int64_t o = sc.off[j];
    bool cp = sc.couple[j] != 0;
    for (int t = threadIdx.x; t < 2 * Pj; t += blockDim.x) {
        cplx v = x[o + t];
        if (cp) {
            cplx sum = mk(0, 0);
            for (int c = 0; c < slabs; ++c) sum = sum + partial[(size_t)c * n_unk + o + t];
            int tt = t < Pj ? t : t - Pj;
            int n, m;
            decode_nm(tt, n, m);
            cplx tm = (t < Pj) ? sc.an[(size_t)j * sc.pmax + n - 1] : sc.bn[(size_t)j * sc.pmax + n - 1];
            v = v + tm * sum;
        }
        y[o + t] = v;
    }
}

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
