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
// One CTA owns one target sphere j and a strided subset of the sources (blockIdx.y); its
// partial sum goes to a per-chunk slab that k_direct_finish adds in a fixed order, so results
// are bit-reproducible.
#include "foggy_kernels.cuh"
#include "k_special.cuh"

namespace foggy {

namespace {
constexpr int kThreads = 256;

__device__ __forceinline__ cplx ipow_mul(int p, cplx c) {
    switch (p & 3) {
        case 0: return c;
        case 1: return mk(-c.y, c.x);
        case 2: return mk(-c.x, -c.y);
        default: return mk(c.y, -c.x);
    }
}
__device__ __forceinline__ void decode_nm(int t, int& n, int& m) {
    int nn = (int)sqrt((double)(t + 1));
    if ((nn + 1) * (nn + 1) <= t + 1) ++nn;
    if (nn * nn > t + 1) --nn;
    n = nn;
    m = t + 1 - nn * nn - nn;
}
__device__ __forceinline__ void decode_nk(int u, int& n, int& k) {
    int nn = (int)((-1.0 + sqrt(9.0 + 8.0 * u)) * 0.5);
    while ((nn - 1) * (nn + 2) / 2 > u) --nn;
    while (nn * (nn + 3) / 2 <= u) ++nn;
    n = nn;
    k = u - (nn - 1) * (nn + 2) / 2;
}

struct Smem {
    double* dq;
    double* jb;
    double* yb;
    cplx* zeta;
    cplx* eph;
    cplx* xr;
    cplx* yr;
    cplx* acc;
    double* geom;
};

__host__ __device__ inline size_t align2(size_t v) { return (v + 1) & ~(size_t)1; }

__device__ inline Smem carve(double* base, int pmax) {
    Smem s;
    size_t o = 0;
    int P = pmax * (pmax + 2);
    s.dq = base + o;   o += align2(dq_size(pmax));
    s.jb = base + o;   o += align2(2 * pmax + 3);
    s.yb = base + o;   o += align2(2 * pmax + 3);
    s.zeta = reinterpret_cast<cplx*>(base + o); o += 2 * (2 * pmax + 3);
    s.eph = reinterpret_cast<cplx*>(base + o);  o += 2 * (2 * pmax + 1);
    s.xr = reinterpret_cast<cplx*>(base + o);   o += 2 * (2 * P);
    s.yr = reinterpret_cast<cplx*>(base + o);   o += 2 * (2 * P);
    s.acc = reinterpret_cast<cplx*>(base + o);  o += 2 * (2 * P);
    s.geom = base + o;
    return s;
}

// Fills zeta[p] = i^p z_p(rho) for p <= P, e^{i mu phi} for |mu| <= pp and the d-table for
// degrees <= pp.  Warp 0 runs the Bessel recurrences and the phases, the other warps the
// d-table columns; ends with a barrier.
__device__ inline void pair_tables(const Smem& s, double rho, double theta, double phi, int P, int pp, int z,
                                   const double* sqrt_binom, const double* rs, int K) {
    int tid = threadIdx.x;
    int warp = tid >> 5, lane = tid & 31;
    if (warp == 0) {
        if (lane == 0) dev_sph_jn(rho, P, s.jb);
        else if (lane == 1 && z != 1) dev_sph_yn(rho, P, s.yb);
        for (int mu = -pp + lane; mu <= pp; mu += 32) {
            double sn, cs;
            sincos((double)mu * phi, &sn, &cs);
            s.eph[mu + pp] = mk(cs, sn);
        }
    } else {
        // The reference evaluates its Legendre functions at x = cos(theta) with
        // sqrt(|1 - x^2|) as the sine (LPMNS, lib_math_legendre.f90:68-126); the half angles
        // are taken from that same (x, s) so that the rotation sees the angle the reference
        // sees, also where cos(theta) rounds to +-1.
        double cb = cos(theta);
        double sbf = sqrt(fabs(1.0 - cb * cb));
        double sb2, cb2;
        if (cb >= 0.0) {
            cb2 = sqrt(0.5 * (1.0 + cb));
            sb2 = 0.5 * sbf / cb2;
        } else {
            sb2 = sqrt(0.5 * (1.0 - cb));
            cb2 = 0.5 * sbf / sb2;
        }
        int ncol = (pp + 1) * (pp + 1);
        for (int t = tid - 32; t < ncol; t += blockDim.x - 32) {
            int mp = (int)sqrt((double)t);
            if ((mp + 1) * (mp + 1) <= t) ++mp;
            if (mp * mp > t) --mp;
            int m = t - mp * mp - mp;
            dq_column(s.dq, mp, m, pp, cb, cb2, sb2, sqrt_binom, rs, K);
        }
    }
    __syncthreads();
    for (int p = tid; p <= P; p += blockDim.x) {
        cplx zc;
        switch (z) {
            case 1: zc = mk(s.jb[p], 0.0); break;
            case 2: zc = mk(s.yb[p], 0.0); break;
            case 3: zc = mk(s.jb[p], s.yb[p]); break;
            default: zc = mk(s.jb[p], -s.yb[p]); break;
        }
        s.zeta[p] = ipow_mul(p, zc);
    }
}

// axial A_ax(k; n, nu), B_ax(k; n, nu) for k >= 0 from the 3j tables and zeta
__device__ __forceinline__ void axial_coeff(const AxialView& ax, const cplx* zeta, int k, int n, int nu, cplx& A,
                                            cplx& B) {
    int S = ax.pmax + 1;
    int o = ax.offset[((size_t)k * S + n) * S + nu];
    int qm = min(n, nu);
    cplx a = mk(0, 0), b = mk(0, 0);
    const double* ga = ax.ga + o;
    const double* gb = ax.gb + o;
    for (int q = 0; q <= qm; ++q) {
        int p = n + nu - 2 * q;
        double g1 = __ldg(ga + q);
        a.x += g1 * zeta[p].x;
        a.y += g1 * zeta[p].y;
        if (q >= 1) {
            double g2 = __ldg(gb + q);
            b.x += g2 * zeta[p + 1].x;
            b.y += g2 * zeta[p + 1].y;
        }
    }
    A = a;
    B = b;
}

}  // namespace

size_t direct_smem_bytes(int pmax) {
    int P = pmax * (pmax + 2);
    size_t o = 0;
    o += align2(dq_size(pmax));
    o += align2(2 * pmax + 3) * 2;
    o += 2 * (2 * pmax + 3) + 2 * (2 * pmax + 1);
    o += 3 * 2 * (2 * (size_t)P);
    o += 4;
    return o * sizeof(double);
}

__global__ void __launch_bounds__(kThreads) k_direct(DirectArgs a) {
    extern __shared__ double smem_d[];
    const SceneView& sc = a.sc;
    Smem s = carve(smem_d, sc.pmax);
    int j = blockIdx.x;
    int c = blockIdx.y;
    if (!sc.couple[j]) return;
    int tid = threadIdx.x;
    int pj = sc.p[j];
    int Pj = pj * (pj + 2);
    for (int t = tid; t < 2 * Pj; t += blockDim.x) s.acc[t] = mk(0, 0);
    const double* cj = sc.centres + 3 * (size_t)j;

    for (int l = c; l < sc.n; l += a.chunks) {
        if (l == j) continue;
        int pl = sc.p[l];
        int Pl = pl * (pl + 2);
        int pp = max(pj, pl);
        int P = pj + pl + 1;
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
        __syncthreads();
        double rho = s.geom[0], theta = s.geom[1], phi = s.geom[2];
        pair_tables(s, rho, theta, phi, P, pp, a.z, a.sqrt_binom, a.rs, a.K);

        // rotate the source: x'_nu[k] = sum_mu d^nu_{mu k} e^{i mu phi} x_nu[mu]
        const cplx* xl = a.x + sc.off[l];
        for (int t = tid; t < Pl; t += blockDim.x) {
            int nu, k;
            decode_nm(t, nu, k);
            cplx sa = mk(0, 0), sb = mk(0, 0);
            int base = nu * nu - 1 + nu;
            for (int mu = -nu; mu <= nu; ++mu) {
                double dv = dq_get(s.dq, nu, mu, k);
                cplx e = s.eph[mu + pp];
                cplx xa = xl[base + mu], xb = xl[Pl + base + mu];
                sa = sa + dv * (e * xa);
                sb = sb + dv * (e * xb);
            }
            s.xr[t] = sa;
            s.xr[Pl + t] = sb;
        }
        __syncthreads();

        // axial translation, outputs (n, +-k)
        int nout = pj * (pj + 3) / 2;
        for (int u = tid; u < nout; u += blockDim.x) {
            int n, k;
            decode_nk(u, n, k);
            cplx yap = mk(0, 0), ybp = mk(0, 0), yam = mk(0, 0), ybm = mk(0, 0);
            for (int nu = max(k, 1); nu <= pl; ++nu) {
                cplx A, B;
                axial_coeff(a.ax, s.zeta, k, n, nu, A, B);
                int ip = nu * nu - 1 + nu + k;
                cplx xap = s.xr[ip], xbp = s.xr[Pl + ip];
                yap = yap + A * xap + B * xbp;
                ybp = ybp + B * xap + A * xbp;
                if (k > 0) {
                    int im = nu * nu - 1 + nu - k;
                    cplx xam = s.xr[im], xbm = s.xr[Pl + im];
                    yam = yam + A * xam - B * xbm;
                    ybm = ybm - B * xam + A * xbm;
                }
            }
            int op = n * n - 1 + n + k;
            s.yr[op] = yap;
            s.yr[Pj + op] = ybp;
            if (k > 0) {
                int om = n * n - 1 + n - k;
                s.yr[om] = yam;
                s.yr[Pj + om] = ybm;
            }
        }
        __syncthreads();

        // rotate back and accumulate: y_nm += e^{-i m phi} sum_k d^n_{mk} y'_n[k]
        for (int t = tid; t < Pj; t += blockDim.x) {
            int n, m;
            decode_nm(t, n, m);
            cplx sa = mk(0, 0), sb = mk(0, 0);
            int base = n * n - 1 + n;
            for (int k = -n; k <= n; ++k) {
                double dv = dq_get(s.dq, n, m, k);
                sa = sa + dv * s.yr[base + k];
                sb = sb + dv * s.yr[Pj + base + k];
            }
            cplx e = conjg(s.eph[m + pp]);
            s.acc[t] = s.acc[t] + e * sa;
            s.acc[Pj + t] = s.acc[Pj + t] + e * sb;
        }
        __syncthreads();
    }
    cplx* out = a.partial + (size_t)c * a.n_unk + sc.off[j];
    for (int t = tid; t < 2 * Pj; t += blockDim.x) out[t] = s.acc[t];
}

void launch_direct(const DirectArgs& a, cudaStream_t s) {
    size_t smem = direct_smem_bytes(a.sc.pmax);
    cudaFuncSetAttribute(k_direct, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    dim3 grid(a.sc.n, a.chunks);
    k_direct<<<grid, kThreads, smem, s>>>(a);
}

__global__ void k_direct_finish(SceneView sc, const cplx* x, const cplx* partial, int chunks, int64_t n_unk,
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
            for (int c = 0; c < chunks; ++c) sum = sum + partial[(size_t)c * n_unk + o + t];
            int tt = t < Pj ? t : t - Pj;
            int n, m;
            decode_nm(tt, n, m);
            cplx tm = (t < Pj) ? sc.an[(size_t)j * sc.pmax + n - 1] : sc.bn[(size_t)j * sc.pmax + n - 1];
            v = v + tm * sum;
        }
        y[o + t] = v;
    }
}

// A, B of one translation in the scaled basis, row (n, m) major: rows n = 1..pn, columns
// nu = 1..pnu; one CTA.
__global__ void __launch_bounds__(kThreads) k_translation_pair(AxialView ax, const double* sqrt_binom,
                                                               const double* rs, int K, double x, double theta,
                                                               double phi, int pn, int pnu, int z, cplx* A,
                                                               cplx* B) {
    extern __shared__ double smem_t[];
    int pmax = max(pn, pnu);
    Smem s = carve(smem_t, pmax);
    int pp = pmax;
    int P = pn + pnu + 1;
    pair_tables(s, x, theta, phi, P, pp, z, sqrt_binom, rs, K);
    __syncthreads();
    int Pn = pn * (pn + 2), Pnu = pnu * (pnu + 2);
    for (int t = threadIdx.x; t < Pn * Pnu; t += blockDim.x) {
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
