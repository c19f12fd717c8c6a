// Direct sphere-sphere coupling operator (the reference's
// lib_mie_ms_solver_calculate_vector_b_without_transposed_all,
// FoggySim/src/lib/mie_theory/lib_mie_ms_solver_interface.f90:806-998):
//
//   y_j = x_j + diag(a_n, b_n) sum_{l != j} [A x_a + B x_b ; B x_a + A x_b](k (d_l - d_j))
//
// The reference builds the full O(p^4) translation matrices A, B from Wigner-3j sums for every
// pair and every matvec (lib_math_vector_spherical_harmonics.f90:1354-1585).  Here each pair
// applies the same operator in O(p^3), in the basis x_nm / g_nm (g_nm = (-1)^m
// sqrt((n+m)!/(n-m)!)), as rotate -> coaxial translate -> rotate back:
//
//   A(theta, phi)_{nm, nu mu} = e^{i(mu-m)phi} sum_k d^n_{mk}(theta) d^nu_{mu k}(theta) A_ax(k; n, nu).
//
// Rotations.  Every small-d matrix factors through the fixed matrix Delta^j = d^j(pi/2)
// (gaunt.cpp::build_delta_table):
//
//   d^j_{m'm}(theta) = i^{m'-m} sum_s Delta^j_{sm'} e^{-i s theta} Delta^j_{sm},
//
// so a rotation is two products with a geometry-independent table and a diagonal phase, and no
// per-pair d-table is built.  Delta's parity symmetries (Delta_{b,-a} = (-1)^{j+b} Delta_{ba},
// Delta_{-b,a} = (-1)^{j+a} Delta_{ba}) let one thread form both outputs b and -b from the
// (j+1)^2 quarter of the table, with inputs folded as u_a +- u_{-a}.
//
// Coaxial step.  With the scalar coaxial coefficients
//   S(k; n, mu) = sum_p i^p (2p+1) (n mu p; -k k 0)(n mu p; 0 0 0) z_p(k d)
// the vector coefficients are
//   A_ax(k; n, nu) = pre [2 nu(nu+1) S(k;n,nu) + i (c1 S(k;n,nu+1) - c2 S(k;n,nu-1))],
//   B_ax(k; n, nu) = pre 2 i k (k d) S(k;n,nu),
//   pre = (-1)^k (2nu+1)/(2n(n+1)), c1 = kd 2nu sqrt((nu+1)^2-k^2)/(2nu+1),
//   c2 = kd 2(nu+1) sqrt(nu^2-k^2)/(2nu+1),
// so for each order k the translated field is out(n) = (-1)^k/(2n(n+1)) sum_mu S(k;n,mu) w(mu),
// where w(mu) gathers the rotated source at degrees mu-1, mu, mu+1: four complex products per S
// entry give a' and b' at +k and -k.
//
// The a and b parts stay separate throughout: combining them as a +- b would diagonalise the
// axial block but loses the relative precision of the smaller part when |A| >> |B| (large
// Hankel values at small kd), which the FP64 parity with the reference does not allow.
//
// Work decomposition.  Spheres are grouped into buckets of similar truncation order; one launch
// per (target bucket, source bucket) sizes its shared memory for the larger order of the two.
// One CTA owns one target sphere and a strided subset of one source bucket and keeps the
// target's accumulator in shared memory.  Per source pair, seven stages separated by CTA
// barriers (items spread over all threads):
//   1. source x (phase e^{i mu (phi + pi/2)}) folded into u_mu +- u_{-mu}
//   2. Delta u, times e^{-i s theta}, folded for the transposed product
//   3. Delta^T: the rotated source x'(nu, +-k), times (2nu+1)
//   4. w(k, mu) for a' and b' at +k and -k
//   5. out(k, n) = sum_mu S(k; n, mu) w(mu)    (S from the pair tables or the Gaunt sums)
//   6. Delta on the translated field, times e^{-i s theta}
//   7. Delta^T, phase e^{-i m (phi + pi/2)}, added to the accumulator; meanwhile threads
//      prepare the geometry and phase tables of the next source.
// The CTA's partial sum goes to its own slab that k_direct_finish adds in a fixed order, so
// results are bit-reproducible.
#include "k_common.cuh"
#include "k_special.cuh"

namespace foggy {

namespace {
constexpr int kThreads = 256;
constexpr int kPrefetch5 = 4;   // coaxial entries loaded ahead per thread

// offset of degree j in the folded [+ 0..j | - 0..j] layout (2(j+1) entries per degree)
__host__ __device__ __forceinline__ int off2(int j) { return (j - 1) * (j + 2); }
__host__ __device__ __forceinline__ int qoff(int j) { return j * (j + 1) * (2 * j + 1) / 6; }

__host__ __device__ inline int szA(int pp) { return 2 * pp * (pp + 3); }
__host__ __device__ inline int szB(int pp) { return 2 * (pp + 1) * (pp + 4); }
__host__ __device__ inline int szAcc(int pp) { return 2 * pp * (pp + 2); }
__host__ __device__ inline int szZ(int pp) { return 2 * pp + 4; }

// element types of an operator precision: the complex C of its arithmetic and its real R
template <class C>
using real_of = decltype(C::x);
template <class C>
struct Vec2T;
template <>
struct Vec2T<cplx> {
    using type = double2;
};
template <>
struct Vec2T<cplxf> {
    using type = float2;
};

template <class C>
struct Bufs {
    short2* nk;    // [pp (pp + 3) / 2] item u -> (degree, order >= 0)
    C* A;          // folded source (1), rotated source x' (3), folded translated field (5)
    C* B;          // folded rotated source (2), w (4), folded rotated field (6)
    C* acc;        // target accumulator (a | b), standard layout
    C* eps;        // [2][pp + 1] e^{i mu (phi + pi/2)}
    C* eth;        // [2][pp + 1] e^{-i s theta}
    C* zeta;       // [2pp + 4] i^p z_p (no pair tables)
    double* jb;    // [2][2pp + 4]
    double* yb;    // [2][2pp + 4]
    double* rho;   // [2]
};

__host__ __device__ inline int szNK(int pp) { return (pp * (pp + 3) / 2 + 3) & ~3; }

// the radial functions and zeta are only kept when S is summed in the kernel (no pair tables)
template <class C>
__host__ __device__ inline size_t smem_bytes(int pp, bool tabs) {
    size_t c = (size_t)szA(pp) + szB(pp) + szAcc(pp) + 4 * (size_t)(pp + 1) + (tabs ? 0 : szZ(pp));
    size_t d = (tabs ? 0 : 4 * (size_t)szZ(pp)) + 2;
    return c * sizeof(C) + d * sizeof(double) + (size_t)szNK(pp) * sizeof(short2);
}

template <class C>
__device__ inline Bufs<C> carve(double* base, int pp, bool tabs) {
    Bufs<C> s;
    C* c = reinterpret_cast<C*>(base);
    s.A = c;           c += szA(pp);
    s.B = c;           c += szB(pp);
    s.acc = c;         c += szAcc(pp);
    s.eps = c;         c += 2 * (pp + 1);
    s.eth = c;         c += 2 * (pp + 1);
    s.zeta = c;        c += tabs ? 0 : szZ(pp);
    double* d = reinterpret_cast<double*>(c);
    s.jb = d;          d += tabs ? 0 : 2 * szZ(pp);
    s.yb = d;          d += tabs ? 0 : 2 * szZ(pp);
    s.rho = d;         d += 2;
    s.nk = reinterpret_cast<short2*>(d);
    return s;
}

// Packed FP32 (Blackwell fma.rn.f32x2): both components of a complex accumulator in one FMA.
__device__ __forceinline__ float2 f2(cplxf c) { return make_float2(c.x, c.y); }
__device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 bcast(float q) { return make_float2(q, q); }

// Work unit of thread tid in the round that starts at b: rounds alternate direction, so where
// the cost of a unit grows (or falls) with its index -- the rotation stages' items are ordered by
// degree, the coaxial rows by order -- every thread's total evens out across rounds and the
// stage's barrier waits less for its slowest thread.  Which thread computes a unit does not
// change what it computes.
__device__ __forceinline__ int snake(int b, int tid) {
    return b + (((b / kThreads) & 1) ? kThreads - 1 - tid : tid);
}

// r += s w in two fused multiply-adds per component
template <class C>
__device__ __forceinline__ void cmac(real_of<C>& rx, real_of<C>& ry, C s, C w) {
    rx = fma(s.x, w.x, rx);
    rx = fma(-s.y, w.y, rx);
    ry = fma(s.x, w.y, ry);
    ry = fma(s.y, w.x, ry);
}

// sum over mu of S(k; n, mu) w_i(mu) for the four planes i of the coaxial stage (a', b' at +k and
// -k).  FP64: four complex MACs per S entry.  FP32: with P_i = sum Re(S) w_i and Q_i = sum Im(S) w_i
// in packed registers, two fma.rn.f32x2 per plane, and S w_i = (P_i.x - Q_i.y, P_i.y + Q_i.x).
template <class C>
struct Mac4;
template <>
struct Mac4<cplx> {
    double r0x = 0, r0y = 0, r1x = 0, r1y = 0, r2x = 0, r2y = 0, r3x = 0, r3y = 0;
    __device__ __forceinline__ void add(cplx S, cplx w0, cplx w1, cplx w2, cplx w3) {
        cmac(r0x, r0y, S, w0);
        cmac(r1x, r1y, S, w1);
        cmac(r2x, r2y, S, w2);
        cmac(r3x, r3y, S, w3);
    }
    __device__ __forceinline__ cplx get(int i) const {
        return i == 0 ? cplx{r0x, r0y} : i == 1 ? cplx{r1x, r1y} : i == 2 ? cplx{r2x, r2y} : cplx{r3x, r3y};
    }
};
template <>
struct Mac4<cplxf> {
    float2 P[4], Q[4];
    __device__ __forceinline__ Mac4() {
#pragma unroll
        for (int i = 0; i < 4; ++i) P[i] = Q[i] = make_float2(0.f, 0.f);
    }
    __device__ __forceinline__ void add(cplxf S, cplxf w0, cplxf w1, cplxf w2, cplxf w3) {
        const float2 sx = bcast(S.x), sy = bcast(S.y);
        P[0] = ffma2(sx, f2(w0), P[0]);
        Q[0] = ffma2(sy, f2(w0), Q[0]);
        P[1] = ffma2(sx, f2(w1), P[1]);
        Q[1] = ffma2(sy, f2(w1), Q[1]);
        P[2] = ffma2(sx, f2(w2), P[2]);
        Q[2] = ffma2(sy, f2(w2), Q[2]);
        P[3] = ffma2(sx, f2(w3), P[3]);
        Q[3] = ffma2(sy, f2(w3), Q[3]);
    }
    __device__ __forceinline__ cplxf get(int i) const { return cplxf{P[i].x - Q[i].y, P[i].y + Q[i].x}; }
};

// Where a translation points: t = k (sign (c_src - c_tgt) + shift).  The direct operator uses
// sign = 1, shift = 0 (t = k (d_l - d_j), the reference's d_j_l); the ML-FMM passes follow the
// reference's own choices per pass.
struct Disp {
    const double* ct;   // target centre
    const double* cs;   // source centre
    double k, sign;
    double sh[3];
};

// The scaled displacement d = k (sign (c_s - c_t) + sh) of a translation and its length, rounded
// the same way wherever it is computed (the translations, and the ML-FMM table set-up that keys
// its coaxial blocks by this length).
__device__ __forceinline__ double disp_vec(const Disp& g, double& d0, double& d1, double& d2) {
    d0 = __dmul_rn(g.k, __fma_rn(g.sign, __dsub_rn(g.cs[0], g.ct[0]), g.sh[0]));
    d1 = __dmul_rn(g.k, __fma_rn(g.sign, __dsub_rn(g.cs[1], g.ct[1]), g.sh[1]));
    d2 = __dmul_rn(g.k, __fma_rn(g.sign, __dsub_rn(g.cs[2], g.ct[2]), g.sh[2]));
    return sqrt(__fma_rn(d0, d0, __fma_rn(d1, d1, __dmul_rn(d2, d2))));
}

// Geometry of one translation and the phase tables of buffer b, spread over fixed threads:
// tid <= pq the azimuthal phases, 64 <= tid <= 64 + pq the polar ones, 100/101 the Bessel
// functions (only without pair tables), the last thread the distance; with a coaxial block
// (sblock), 32..63 prefetch its rows into L2.
template <class C>
__device__ inline void prep_pair(const Bufs<C>& s, const Disp& g, int z, const C* sblock, int pj, int pl, int pp,
                                 int b, int tid, bool bessel) {
    const int pq = max(pj, pl);
    const bool e1 = tid <= pq;
    const bool e2 = tid >= 64 && tid - 64 <= pq;
    const bool e3 = bessel && (tid == 100 || (tid == 101 && z != 1));
    const bool e4 = tid == kThreads - 1;
    if (sblock && tid >= 32 && tid < 64) {
        // rows mu = k..pl+1 of each order's square block, read by the coaxial stage of that pair
        const int M2 = pq + 2;
        for (int k = tid - 32; k <= min(pj, pl); k += 32) {
            // the bulk prefetch takes a 16-byte aligned address and a multiple of 16 bytes: the
            // range is narrowed to the aligned part inside the rows (single-precision entries are
            // 8 bytes)
            const uintptr_t b0 = reinterpret_cast<uintptr_t>(sblock + pair_block_offset(k, M2, M2));
            const uintptr_t b1 = b0 + (uintptr_t)(pl + 2 - k) * (M2 - k) * sizeof(C);
            const uintptr_t a0 = (b0 + 15) & ~(uintptr_t)15, a1 = b1 & ~(uintptr_t)15;
            if (a1 > a0) {
                const unsigned bytes = (unsigned)(a1 - a0);
                asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a0), "r"(bytes) : "memory");
            }
        }
    }
    if (!(e1 || e2 || e3 || e4)) return;
    double d0, d1, d2;
    const double r = disp_vec(g, d0, d1, d2);
    if (e1) {
        const double ph = (d0 == 0.0 && d1 == 0.0) ? 0.0 : atan2(d1, d0);
        double sn, cs;
        sincos((double)tid * ph, &sn, &cs);
        s.eps[b * (pp + 1) + tid] = ipow_mul(tid, cm<C>(cs, sn));
    }
    if (e2) {
        // the reference evaluates its Legendre functions at x = cos(theta) with sqrt(|1 - x^2|) as
        // the sine (LPMNS, lib_math_legendre.f90:68-126); the rotation uses the angle of that
        // same (x, s), which also snaps to 0 or pi where cos(theta) rounds to +-1
        const double th = (r == 0.0) ? 0.0 : acos(d2 / r);
        const double cb = cos(th);
        const double te = atan2(sqrt(fabs(1.0 - cb * cb)), cb);
        const int sidx = tid - 64;
        double sn, cs;
        sincos((double)sidx * te, &sn, &cs);
        s.eth[b * (pp + 1) + sidx] = cm<C>(cs, -sn);
    }
    if (e3) {
        const int P = pj + pl + 1;
        if (tid == 100) dev_sph_jn(r, P, s.jb + b * szZ(pp));
        else dev_sph_yn(r, P, s.yb + b * szZ(pp));
    }
    if (e4) s.rho[b] = r;
}

// The FP32 Delta sums with packed FMAs: each real table entry scales a complex value, so one
// fma.rn.f32x2 does the two real multiply-adds of the scalar form (same roundings, half the
// instructions).  u[a STRIDE] for a = 0..amax.
template <int STRIDE>
__device__ __forceinline__ void delta_sum_f2(const float* __restrict__ Q, int j, int o, int amax, const cplxf* ua,
                                             const cplxf* ub, cplxf& Ea, cplxf& Oa, cplxf& Eb, cplxf& Ob) {
    float2 ea = make_float2(0.f, 0.f), oa = ea, eb = ea, ob = ea;
    const int st = j + 1;
    int a = 0;
    for (; a + 1 <= amax; a += 2) {
        const float2 q0 = bcast(__ldg(Q + a * st + o));
        const float2 q1 = bcast(__ldg(Q + (a + 1) * st + o));
        ea = ffma2(q0, f2(ua[a * STRIDE]), ea);
        oa = ffma2(q1, f2(ua[(a + 1) * STRIDE]), oa);
        eb = ffma2(q0, f2(ub[a * STRIDE]), eb);
        ob = ffma2(q1, f2(ub[(a + 1) * STRIDE]), ob);
    }
    if (a <= amax) {
        const float2 q0 = bcast(__ldg(Q + a * st + o));
        ea = ffma2(q0, f2(ua[a * STRIDE]), ea);
        eb = ffma2(q0, f2(ub[a * STRIDE]), eb);
    }
    Ea = cplxf{ea.x, ea.y};
    Oa = cplxf{oa.x, oa.y};
    Eb = cplxf{eb.x, eb.y};
    Ob = cplxf{ob.x, ob.y};
}

// E = sum over even a, O = sum over odd a of Q[a (j+1) + o] u[a], a = 0..amax, for the two parts
template <class C>
__device__ __forceinline__ void delta_sum(const real_of<C>* __restrict__ Q, int j, int o, int amax, const C* ua,
                                          const C* ub, C& Ea, C& Oa, C& Eb, C& Ob) {
    if constexpr (sizeof(C) == 8) {
        delta_sum_f2<1>(Q, j, o, amax, ua, ub, Ea, Oa, Eb, Ob);
    } else {
    using R = real_of<C>;
    R eax = 0, eay = 0, oax = 0, oay = 0, ebx = 0, eby = 0, obx = 0, oby = 0;
    const int st = j + 1;
    int a = 0;
    for (; a + 1 <= amax; a += 2) {
        const R q0 = __ldg(Q + a * st + o);
        const R q1 = __ldg(Q + (a + 1) * st + o);
        const C u0 = ua[a], u1 = ua[a + 1], v0 = ub[a], v1 = ub[a + 1];
        eax += q0 * u0.x;
        eay += q0 * u0.y;
        oax += q1 * u1.x;
        oay += q1 * u1.y;
        ebx += q0 * v0.x;
        eby += q0 * v0.y;
        obx += q1 * v1.x;
        oby += q1 * v1.y;
    }
    if (a <= amax) {
        const R q0 = __ldg(Q + a * st + o);
        const C u0 = ua[a], v0 = ub[a];
        eax += q0 * u0.x;
        eay += q0 * u0.y;
        ebx += q0 * v0.x;
        eby += q0 * v0.y;
    }
    Ea = C{eax, eay};
    Oa = C{oax, oay};
    Eb = C{ebx, eby};
    Ob = C{obx, oby};
    }
}

// stages 2 and 6: W = Delta u at +-s, times e^{-+i s theta}; stored folded for the transposed
// product as V = (-1)^s (W'_s +- W'_{-s}) at off2(j) + s and off2(j) + j + 1 + s
template <class C>
__device__ __forceinline__ void fwd_item(const real_of<C>* delta, const C* src, C* dst, int SP, int j, int s_,
                                         int amax, C eth) {
    const int fold = ((j + s_) & 1) ? j + 1 : 0;
    const C* ua = src + off2(j) + fold;
    C Ea, Oa, Eb, Ob;
    delta_sum(delta + qoff(j), j, s_, amax, ua, ua + SP, Ea, Oa, Eb, Ob);
    const real_of<C> pj_ = sgn(j), ps = sgn(s_);
    C* d = dst + off2(j);
#pragma unroll
    for (int part = 0; part < 2; ++part) {
        const C E = part ? Eb : Ea, O = part ? Ob : Oa;
        const C wp = eth * (E + O);
        if (s_ == 0) {
            d[part * SP] = wp;
            d[part * SP + j + 1] = wp;
        } else {
            const C wm = conjg(eth) * (pj_ * (E - O));
            d[part * SP + s_] = ps * (wp + wm);
            d[part * SP + j + 1 + s_] = ps * (wp - wm);
        }
    }
}
// Shared-memory buffers and tables of one CTA's translations.
template <class C>
struct PairCtx {
    Bufs<C> s;
    const real_of<C>* delta;   // d^j(pi/2)
    DTabs dt;              // rs[j][k] = sqrt(j^2 - k^2)
    SGaunt g;              // scalar Gaunt sums (no coaxial block)
    int z;                 // radial function of the translation
    int pp, SP, XP;        // largest degree; part strides of the folded buffers and of x'
    bool tabs;             // coaxial blocks given (else S is summed from the Gaunt table)
};

// One translation (target degree pj <- source degree pl, source coefficients xl, scaled basis)
// added into c.s.acc: the seven stages with their barriers.  Its geometry and phase tables
// were prepared in buffer cur; next(tid) prepares the following translation into the other
// buffer while the last stage runs.  Coincident centres (distance 0) add the source unchanged,
// as the reference does for them.
template <class C, class Next>
__device__ inline void run_pair(const PairCtx<C>& c, int tid, int pj, int pl, const cplx* __restrict__ xl,
                                const C* pair_s, int cur, Next next) {
    using R = real_of<C>;
    using V2 = typename Vec2T<C>::type;
    const Bufs<C>& s = c.s;
    const R* delta = c.delta;
    const int pp = c.pp, SP = c.SP, XP = c.XP;
    const bool tabs = c.tabs;
    const int Pj = pj * (pj + 2);
    if (s.rho[cur] == 0.0) {
        const int pm = min(pj, pl), Pm = pm * (pm + 2), Pl = pl * (pl + 2);
        for (int t = tid; t < 2 * Pm; t += kThreads) {
            const int part = t >= Pm, e = t - part * Pm;
            s.acc[part * Pj + e] = s.acc[part * Pj + e] + cm<C>(xl[part * Pl + e].x, xl[part * Pl + e].y);
        }
        next(tid);
        __syncthreads();
        return;
    }
    const int Pl = pl * (pl + 2);
    const int kmax = min(pj, pl);
    const C* eps = s.eps + cur * (pp + 1);
    const C* eth = s.eth + cur * (pp + 1);
    // ---- 1. u = e^{i mu (phi + pi/2)} x, folded ------------------------------------------
    {
        const int items = pl * (pl + 3) / 2;
        for (int t = tid; t < items; t += kThreads) {
            const short2 d_ = s.nk[t];
            const int nu = d_.x, mu = d_.y;
            const int base = nu * nu - 1 + nu;
            const C e = eps[mu];
            C* U = s.A + off2(nu) + mu;
            // the four source entries are all in flight before any use
            const double2* xv = reinterpret_cast<const double2*>(xl + base);
            const double2 ap = __ldcg(xv + mu), am = __ldcg(xv - mu);
            const double2 bp = __ldcg(xv + Pl + mu), bm = __ldcg(xv + Pl - mu);
            const C ua = e * cm<C>(ap.x, ap.y), ub = e * cm<C>(bp.x, bp.y);
            if (mu == 0) {
                U[0] = ua;
                U[nu + 1] = ua;
                U[SP] = ub;
                U[SP + nu + 1] = ub;
            } else {
                const C va = conjg(e) * cm<C>(am.x, am.y), vb = conjg(e) * cm<C>(bm.x, bm.y);
                U[0] = ua + va;
                U[nu + 1] = ua - va;
                U[SP] = ub + vb;
                U[SP + nu + 1] = ub - vb;
            }
        }
        if (!tabs) {
            const int P = pj + pl + 1;
            const double* jb = s.jb + cur * szZ(pp);
            const double* yb = s.yb + cur * szZ(pp);
            for (int p = tid; p <= P; p += kThreads) {
                const cplx z = zeta_of(c.z, p, jb, yb);
                s.zeta[p] = cm<C>(z.x, z.y);
            }
        }
    }
    __syncthreads();
    // ---- 2. Delta u, e^{-i s theta} ----------------------------------------------------------
    {
        const int items = pl * (pl + 3) / 2;
        for (int b_ = 0; b_ < items; b_ += kThreads) {
            const int t = snake(b_, tid);
            if (t >= items) continue;
            const short2 d_ = s.nk[t];
            const int nu = d_.x, s_ = d_.y;
            fwd_item(delta, s.A, s.B, SP, nu, s_, nu, eth[s_]);
        }
    }
    __syncthreads();
    // ---- 3. Delta^T: x'(nu, +-k) = i^{+-k} T_{+-k}, stored times (2nu+1) ------------------
    {
        const int items = pl * (pl + 3) / 2;
        for (int b_ = 0; b_ < items; b_ += kThreads) {
            const int t = snake(b_, tid);
            if (t >= items) continue;
            const short2 d_ = s.nk[t];
            const int nu = d_.x, k = d_.y;
            const int fold = ((nu + k) & 1) ? nu + 1 : 0;
            const C* va = s.B + off2(nu) + fold;
            C Ea, Oa, Eb, Ob;
            delta_sum(delta + qoff(nu), nu, k, nu, va, va + SP, Ea, Oa, Eb, Ob);
            const R f = 2.0 * nu + 1.0;
            const R pn = sgn(nu);
            C* X = s.A + nu * nu - 1 + nu;
#pragma unroll
            for (int part = 0; part < 2; ++part) {
                const C E = part ? Eb : Ea, O = part ? Ob : Oa;
                X[part * XP + k] = ipow_mul(k, f * (E + O));
                if (k > 0) X[part * XP - k] = ipow_mul(-k, (f * pn) * (E - O));
            }
        }
    }
    __syncthreads();
    // ---- 4. w(k, mu) for a', b' at +k and -k ---------------------------------------------
    {
        const double x = s.rho[cur];
        const int items = (kmax + 1) * (pl + 2) - kmax * (kmax + 1) / 2;
        const int W = c.dt.K + 1;
        for (int t = tid; t < items; t += kThreads) {
            int k = 0, rem = t;
            while (rem >= pl + 2 - k) {
                rem -= pl + 2 - k;
                ++k;
            }
            const int mu = k + rem;
            const int lo = max(1, k);
            const R c0 = 2.0 * mu * (mu + 1.0);
            const R c1m = (mu - 1 >= lo) ? x * 2.0 * (mu - 1) * c.dt.rs[mu * W + k] / (2.0 * mu - 1.0) : 0.0;
            const R c2p = (mu + 1 <= pl) ? x * 2.0 * (mu + 2) * c.dt.rs[(mu + 1) * W + k] / (2.0 * mu + 3.0) : 0.0;
            const R bk2 = 2.0 * k * x;
            C* w = s.B + t;   // four planes of `items` entries: a'(+k), b'(+k), a'(-k), b'(-k)
#pragma unroll
            for (int sg = 0; sg < 2; ++sg) {
                const int kk = sg ? -k : k;
                const R bs = sg ? -bk2 : bk2;
                C av[3], bv[3];
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    const int nu = mu - 1 + d;
                    const bool ok = nu >= lo && nu <= pl;
                    const int o = nu * nu - 1 + nu + kk;
                    av[d] = ok ? s.A[o] : C{0, 0};
                    bv[d] = ok ? s.A[XP + o] : C{0, 0};
                }
                // wa = c0 a + i (bs b + c1m a_- - c2p a_+),  wb = c0 b + i (bs a + c1m b_- - c2p b_+)
                const C ia = bs * bv[1] + c1m * av[0] - c2p * av[2];
                const C ib = bs * av[1] + c1m * bv[0] - c2p * bv[2];
                w[2 * sg * items] = C{c0 * av[1].x - ia.y, c0 * av[1].y + ia.x};
                w[(2 * sg + 1) * items] = C{c0 * bv[1].x - ib.y, c0 * bv[1].y + ib.x};
            }
        }
    }
    __syncthreads();
    // ---- 5. out(k, n) = sum_mu S(k; n, mu) w(k, mu), folded for the back rotation ----------
    {
        // rows(k) = pj - max(1, k) + 1: k = 0 and k = 1 both have pj rows
        const int rows_tot = pj + (kmax >= 1 ? kmax * pj - (kmax - 1) * kmax / 2 : 0);
        const int NW = (kmax + 1) * (pl + 2) - kmax * (kmax + 1) / 2;   // w plane stride
        const int M2 = max(pj, pl) + 2;
        for (int b_ = 0; b_ < rows_tot; b_ += kThreads) {
            const int t = snake(b_, tid);
            if (t >= rows_tot) continue;
            int k = 0, rem = t;
            for (;;) {
                const int rk = pj - max(1, k) + 1;
                if (rem < rk) break;
                rem -= rk;
                ++k;
            }
            const int n = max(1, k) + rem;
            const C* w = s.B + (k * (pl + 2) - k * (k - 1) / 2);
            const int cnt = pl + 2 - k;
            // FP32: packed FMAs (Mac4); FP64: four scalar complex MACs per S entry
            C a0, a1, a2, a3;
            if constexpr (sizeof(C) == 8) {
                Mac4<C> acc;
                if (tabs) {
                    const int Wk = M2 - k;
                    const V2* sp = reinterpret_cast<const V2*>(pair_s + pair_block_offset(k, M2, M2) + (n - k));
                    // kPrefetch5 coaxial entries in flight per thread: the rows come from L2, so the loop
                    // is bounded by how many loads overlap, not by the multiply-adds
                    int q = 0;
                    for (; q + kPrefetch5 <= cnt; q += kPrefetch5) {
                        V2 sv[kPrefetch5];
    #pragma unroll
                        for (int u = 0; u < kPrefetch5; ++u) sv[u] = __ldcg(sp + (q + u) * Wk);
    #pragma unroll
                        for (int u = 0; u < kPrefetch5; ++u)
                            acc.add(C{sv[u].x, sv[u].y}, w[q + u], w[NW + q + u], w[2 * NW + q + u], w[3 * NW + q + u]);
                    }
                    for (; q < cnt; ++q) {
                        const V2 sv = __ldcg(sp + q * Wk);
                        acc.add(C{sv.x, sv.y}, w[q], w[NW + q], w[2 * NW + q], w[3 * NW + q]);
                    }
                } else {
                    const int W = c.g.NM - k + 1;
                    const size_t plane = (size_t)W * W;
                    const double* G = c.g.gs + c.g.koff[k] + (n - k);
                    for (int q = 0; q < cnt; ++q) {
                        const int mu = k + q;
                        const double* gp = G + (size_t)(mu - k) * W;
                        const int qm = min(n, mu);
                        int p = n + mu;
                        double sx = 0.0, sy = 0.0;
                        for (int qq = 0; qq <= qm; ++qq, p -= 2) {
                            const double gq = __ldg(gp + qq * plane);
                            sx += gq * s.zeta[p].x;
                            sy += gq * s.zeta[p].y;
                        }
                        acc.add(cm<C>(sx, sy), w[q], w[NW + q], w[2 * NW + q], w[3 * NW + q]);
                    }
                }
                a0 = acc.get(0);
                a1 = acc.get(1);
                a2 = acc.get(2);
                a3 = acc.get(3);
            } else {
                R r0x = 0, r0y = 0, r1x = 0, r1y = 0, r2x = 0, r2y = 0, r3x = 0, r3y = 0;
                if (tabs) {
                    const int Wk = M2 - k;
                    const V2* sp = reinterpret_cast<const V2*>(pair_s + pair_block_offset(k, M2, M2) + (n - k));
                    // kPrefetch5 coaxial entries in flight per thread: the rows come from L2, so the loop
                    // is bounded by how many loads overlap, not by the multiply-adds
                    int q = 0;
                    for (; q + kPrefetch5 <= cnt; q += kPrefetch5) {
                        V2 sv[kPrefetch5];
    #pragma unroll
                        for (int u = 0; u < kPrefetch5; ++u) sv[u] = __ldcg(sp + (q + u) * Wk);
    #pragma unroll
                        for (int u = 0; u < kPrefetch5; ++u) {
                            const C S = C{sv[u].x, sv[u].y};
                            cmac(r0x, r0y, S, w[q + u]);
                            cmac(r1x, r1y, S, w[NW + q + u]);
                            cmac(r2x, r2y, S, w[2 * NW + q + u]);
                            cmac(r3x, r3y, S, w[3 * NW + q + u]);
                        }
                    }
                    for (; q < cnt; ++q) {
                        const V2 sv = __ldcg(sp + q * Wk);
                        const C S = C{sv.x, sv.y};
                        cmac(r0x, r0y, S, w[q]);
                        cmac(r1x, r1y, S, w[NW + q]);
                        cmac(r2x, r2y, S, w[2 * NW + q]);
                        cmac(r3x, r3y, S, w[3 * NW + q]);
                    }
                } else {
                    const int W = c.g.NM - k + 1;
                    const size_t plane = (size_t)W * W;
                    const double* G = c.g.gs + c.g.koff[k] + (n - k);
                    for (int q = 0; q < cnt; ++q) {
                        const int mu = k + q;
                        const double* gp = G + (size_t)(mu - k) * W;
                        const int qm = min(n, mu);
                        int p = n + mu;
                        double sx = 0.0, sy = 0.0;
                        for (int qq = 0; qq <= qm; ++qq, p -= 2) {
                            const double gq = __ldg(gp + qq * plane);
                            sx += gq * s.zeta[p].x;
                            sy += gq * s.zeta[p].y;
                        }
                        const C S = cm<C>(sx, sy);
                        cmac(r0x, r0y, S, w[q]);
                        cmac(r1x, r1y, S, w[NW + q]);
                        cmac(r2x, r2y, S, w[2 * NW + q]);
                        cmac(r3x, r3y, S, w[3 * NW + q]);
                    }
                }
                a0 = C{r0x, r0y};
                a1 = C{r1x, r1y};
                a2 = C{r2x, r2y};
                a3 = C{r3x, r3y};
            }
            const R f = sgn(k) / (2.0 * n * (n + 1.0));
            C* U = s.A + off2(n) + k;
            if (k == 0) {
                U[0] = f * a0;
                U[n + 1] = U[0];
                U[SP] = f * a1;
                U[SP + n + 1] = U[SP];
            } else {
                // u'_{+k} = i^{-k} y'(+k), u'_{-k} = i^{k} y'(-k)
                const C ap = ipow_mul(-k, f * a0), am = ipow_mul(k, f * a2);
                const C bp = ipow_mul(-k, f * a1), bm = ipow_mul(k, f * a3);
                U[0] = ap + am;
                U[n + 1] = ap - am;
                U[SP] = bp + bm;
                U[SP + n + 1] = bp - bm;
            }
        }
    }
    __syncthreads();
    // ---- 6. Delta on the translated field, e^{-i s theta} (orders |k| <= kmax only) ----------
    {
        const int items = pj * (pj + 3) / 2;
        for (int b_ = 0; b_ < items; b_ += kThreads) {
            const int t = snake(b_, tid);
            if (t >= items) continue;
            const short2 d_ = s.nk[t];
            const int n = d_.x, s_ = d_.y;
            fwd_item(delta, s.A, s.B, SP, n, s_, min(n, kmax), eth[s_]);
        }
    }
    __syncthreads();
    // ---- 7. Delta^T, phase, accumulate; then the next pair's tables ---------------------------
    {
        const int items = pj * (pj + 3) / 2;
        for (int b_ = 0; b_ < items; b_ += kThreads) {
            const int t = snake(b_, tid);
            if (t >= items) continue;
            const short2 d_ = s.nk[t];
            const int n = d_.x, m = d_.y;
            const int fold = ((n + m) & 1) ? n + 1 : 0;
            const C* va = s.B + off2(n) + fold;
            C Ea, Oa, Eb, Ob;
            delta_sum(delta + qoff(n), n, m, n, va, va + SP, Ea, Oa, Eb, Ob);
            const R pn = sgn(n);
            const C e = eps[m];
            C* acc = s.acc + n * n - 1 + n;
#pragma unroll
            for (int part = 0; part < 2; ++part) {
                const C E = part ? Eb : Ea, O = part ? Ob : Oa;
                acc[part * Pj + m] = acc[part * Pj + m] + conjg(e) * (E + O);
                if (m > 0) acc[part * Pj - m] = acc[part * Pj - m] + e * (pn * (E - O));
            }
        }
        next(tid);
    }
    __syncthreads();
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

// ---------------------------------------------------------------------------------------------
// the pair tables and the d(pi/2) table of an operator precision
__device__ __forceinline__ const cplx* stab_of(const DirectArgs& a, cplx*) { return a.pt.stab; }
template <class C>
__host__ inline const C* stab_of_host(const DirectArgs& a);
template <>
__host__ inline const cplx* stab_of_host<cplx>(const DirectArgs& a) { return a.pt.stab; }
template <>
__host__ inline const cplxf* stab_of_host<cplxf>(const DirectArgs& a) { return a.pt.stab32; }
__device__ __forceinline__ const cplxf* stab_of(const DirectArgs& a, cplxf*) { return a.pt.stab32; }
__device__ __forceinline__ const double* delta_of(const DirectArgs& a, cplx*) { return a.delta; }
__device__ __forceinline__ const float* delta_of(const DirectArgs& a, cplxf*) { return a.delta32; }

// CTAs per SM the register budget is set for: the FP64 operator needs 80 registers a thread
// (3 CTAs); the FP32 one fits 64 without spills, so 4 CTAs where shared memory allows
// (orders up to 28)
template <class C>
struct DirectOcc {
    static constexpr int ctas = 3;
};
template <>
struct DirectOcc<cplxf> {
    static constexpr int ctas = 4;
};

template <class C>
__global__ void __launch_bounds__(kThreads, DirectOcc<C>::ctas) k_direct(DirectArgs a, DirectBucket bk) {
    extern __shared__ __align__(16) double smem_d[];
    const SceneView& sc = a.sc;
    const int pp = bk.pp;
    const C* stab = stab_of(a, (C*)nullptr);
    const bool tabs = stab != nullptr;
    const Bufs<C> s = carve<C>(smem_d, pp, tabs);
    const int j = bk.targets[blockIdx.x];
    const int c = blockIdx.y;
    if (!sc.couple[j]) return;
    const int tid = threadIdx.x;
    const int pj = sc.p[j];
    const int Pj = pj * (pj + 2);
    const int SP = pp * (pp + 3);   // part stride of the folded buffers
    const int XP = pp * (pp + 2);   // part stride of x'
    const PairCtx<C> ctx{s, delta_of(a, (C*)nullptr), a.dt, a.g, a.z, pp, SP, XP, tabs};
    for (int t = tid; t < 2 * Pj; t += kThreads) s.acc[t] = C{0, 0};
    for (int t = tid; t < pp * (pp + 3) / 2; t += kThreads) {
        int n, k;
        decode_nk(t, n, k);
        s.nk[t] = make_short2((short)n, (short)k);
    }

    auto block = [&](int l) -> const C* {
        return tabs ? stab + a.pt.pair_off[pair_index(min(j, l), max(j, l), sc.n)] : nullptr;
    };
    auto disp = [&](int l) {
        return Disp{sc.centres + 3 * (size_t)j, sc.centres + 3 * (size_t)l, sc.k, 1.0, {0.0, 0.0, 0.0}};
    };
    int i = c;
    if (i < bk.nsources && bk.sources[i] == j) i += bk.chunks;
    if (i < bk.nsources) {
        const int l = bk.sources[i];
        prep_pair(s, disp(l), a.z, block(l), pj, sc.p[l], pp, 0, tid, !tabs);
    }
    __syncthreads();
    int cur = 0;
    while (i < bk.nsources) {
        const int l = bk.sources[i];
        int inext = i + bk.chunks;
        if (inext < bk.nsources && bk.sources[inext] == j) inext += bk.chunks;
        run_pair(ctx, tid, pj, sc.p[l], a.x + sc.off[l], block(l), cur, [&](int t) {
            if (inext < bk.nsources) {
                const int ln = bk.sources[inext];
                prep_pair(s, disp(ln), a.z, block(ln), pj, sc.p[ln], pp, cur ^ 1, t, !tabs);
            }
        });
        cur ^= 1;
        i = inext;
    }
    cplx* out = a.partial + (size_t)(bk.slab + c) * a.n_unk + sc.off[j];
    for (int t = tid; t < 2 * Pj; t += kThreads) out[t] = mk(s.acc[t].x, s.acc[t].y);
    // slabs of this source bucket that launches with fewer chunks leave unused
    if (c == bk.chunks - 1)
        for (int e = c + 1; e < a.cmax; ++e) {
            cplx* z = a.partial + (size_t)(bk.slab + e) * a.n_unk + sc.off[j];
            for (int t = tid; t < 2 * Pj; t += kThreads) z[t] = mk(0, 0);
        }
}

size_t direct_smem_bytes(int pp, bool tabs, bool fp32) {
    return fp32 ? smem_bytes<cplxf>(pp, tabs) : smem_bytes<cplx>(pp, tabs);
}

void launch_direct(const DirectArgs& a, const DirectBucket& b, cudaStream_t s) {
    dim3 grid(b.ntargets, b.chunks);
    if (a.fp32) {
        size_t smem = direct_smem_bytes(b.pp, a.pt.stab32 != nullptr, true);
        raise_smem_ceiling(reinterpret_cast<const void*>(k_direct<cplxf>), smem);
        k_direct<cplxf><<<grid, kThreads, smem, s>>>(a, b);
    } else {
        size_t smem = direct_smem_bytes(b.pp, a.pt.stab != nullptr, false);
        raise_smem_ceiling(reinterpret_cast<const void*>(k_direct<cplx>), smem);
        k_direct<cplx><<<grid, kThreads, smem, s>>>(a, b);
    }
}


// ---------------------------------------------------------------------------------------------
// ML-FMM passes: CTAs (target, chunk) over the target's CSR source list, chunk c taking the sources
// c, c + chunks, ... of the list; the same seven stages per source, S summed from the Gaunt table
// (the displacements are box geometry, so no pair tables).  With one chunk the result is written to
// (or added onto) the target's coefficients; with several, each chunk writes its partial sum to its
// slab and k_translate_sum adds the slabs in chunk order.
template <class C>
__global__ void __launch_bounds__(kThreads, 3) k_translate(TransArgs a) {
    extern __shared__ __align__(16) double smem_d[];
    const int pp = a.pp;
    const Bufs<C> s = carve<C>(smem_d, pp, false);
    const int t = a.tbase + blockIdx.x;
    const int tid = threadIdx.x;
    const int pj = a.tgt.p[t];
    const int Pj = pj * (pj + 2);
    const int SP = pp * (pp + 3);
    const int XP = pp * (pp + 2);
    const bool tabs = a.tab_off != nullptr;
    const C* tab;
    const real_of<C>* delta;
    if constexpr (sizeof(C) == 8) {
        tab = a.tab32;
        delta = a.delta32;
    } else {
        tab = a.tab;
        delta = a.delta;
    }
    const PairCtx<C> ctx{s, delta, a.dt, a.g, a.z, pp, SP, XP, tabs};
    auto block = [&](int i) -> const C* { return tabs ? tab + a.tab_off[i] : nullptr; };
    const int c = blockIdx.y, chunks = gridDim.y;
    cplx* out = chunks == 1 ? a.out + a.tgt.off[t]
                            : a.slab + ((size_t)c * gridDim.x + blockIdx.x) * a.slab_ld;
    for (int e = tid; e < 2 * Pj; e += kThreads) s.acc[e] = (a.add && chunks == 1) ? cm<C>(out[e].x, out[e].y) : C{0, 0};
    for (int e = tid; e < pp * (pp + 3) / 2; e += kThreads) {
        int n, k;
        decode_nk(e, n, k);
        s.nk[e] = make_short2((short)n, (short)k);
    }
    const int i0 = a.lptr[blockIdx.x], i1 = a.lptr[blockIdx.x + 1];
    auto disp = [&](int l) {
        return Disp{a.tgt.c + 3 * (size_t)t, a.src.c + 3 * (size_t)l, a.k, a.sign, {a.sh[0], a.sh[1], a.sh[2]}};
    };
    if (i0 + c < i1) {
        const int l = a.lidx[i0 + c];
        prep_pair(s, disp(l), a.z, block(i0 + c), pj, a.src.p[l], pp, 0, tid, !tabs);
    }
    __syncthreads();
    int cur = 0;
    for (int i = i0 + c; i < i1; i += chunks) {
        const int l = a.lidx[i];
        run_pair(ctx, tid, pj, a.src.p[l], a.x + a.src.off[l], block(i), cur, [&](int tt) {
            if (i + chunks < i1) {
                const int ln = a.lidx[i + chunks];
                prep_pair(s, disp(ln), a.z, block(i + chunks), pj, a.src.p[ln], pp, cur ^ 1, tt, !tabs);
            }
        });
        cur ^= 1;
    }
    for (int e = tid; e < 2 * Pj; e += kThreads) out[e] = mk(s.acc[e].x, s.acc[e].y);
}

// The ML-FMM's coaxial blocks: for every entry i of a pass's source lists, the translation's
// length rho (disp_vec, as the pass computes it) and degrees (target, source); one CTA per target.
__global__ void k_fmm_rho(TransArgs a, double* rho, int2* deg) {
    const int t = a.tbase + blockIdx.x;
    const int i0 = a.lptr[blockIdx.x], i1 = a.lptr[blockIdx.x + 1];
    for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
        const int l = a.lidx[i];
        const Disp g{a.tgt.c + 3 * (size_t)t, a.src.c + 3 * (size_t)l, a.k, a.sign, {a.sh[0], a.sh[1], a.sh[2]}};
        double d0, d1, d2;
        rho[i] = disp_vec(g, d0, d1, d2);
        deg[i] = make_int2(a.tgt.p[t], a.src.p[l]);
    }
}

// One coaxial block per distinct (rho, target degree, source degree) of a pass: S(k; mu, n) summed
// from the scalar Gaunt table exactly as the translation stage sums it without tables (radial
// functions to degree p_t + p_s + 1, the same terms in the same order), on the square layout of
// the pair tables; entries the translation never reads (mu > p_s + 1 or n > p_t) are zero.
__global__ void __launch_bounds__(256) k_fmm_tab(const FmmTabEntry* u, SGaunt g, int z, cplx* tab) {
    __shared__ double jb[2 * kMaxDegree + 8], yb[2 * kMaxDegree + 8];
    __shared__ cplx zeta[2 * kMaxDegree + 8];
    const FmmTabEntry e = u[blockIdx.x];
    const int M2 = max(e.pt, e.ps) + 2;
    const int P = e.pt + e.ps + 1;
    const int km = min(e.pt, e.ps);
    const int64_t tot = pair_block_size(e.ps, e.pt);
    cplx* out = tab + e.off;
    if (e.rho == 0.0) {   // coincident centres: the translation adds its source unchanged
        for (int64_t q = threadIdx.x; q < tot; q += blockDim.x) out[q] = mk(0, 0);
        return;
    }
    if (threadIdx.x == 0) dev_sph_jn(e.rho, P, jb);
    if (threadIdx.x == 32 && z != 1) dev_sph_yn(e.rho, P, yb);
    __syncthreads();
    for (int p = threadIdx.x; p <= P; p += blockDim.x) zeta[p] = zeta_of(z, p, jb, yb);
    __syncthreads();
    for (int64_t q = threadIdx.x; q < tot; q += blockDim.x) {
        int k = 0;
        while (k < km && pair_block_offset(k + 1, M2, M2) <= q) ++k;
        const int64_t r = q - pair_block_offset(k, M2, M2);
        const int cols = M2 - k;
        const int mu = k + (int)(r / cols), n = k + (int)(r % cols);
        if (mu > e.ps + 1 || n > e.pt) {
            out[q] = mk(0, 0);
            continue;
        }
        const int W = g.NM - k + 1;
        const size_t plane = (size_t)W * W;
        const double* gp = g.gs + g.koff[k] + (size_t)(mu - k) * W + (n - k);
        const int qm = min(n, mu);
        int p = n + mu;
        double sx = 0.0, sy = 0.0;
        for (int qq = 0; qq <= qm; ++qq, p -= 2) {
            const double gq = __ldg(gp + qq * plane);
            sx += gq * zeta[p].x;
            sy += gq * zeta[p].y;
        }
        out[q] = mk(sx, sy);
    }
}

// single-precision copy of tables
__global__ void k_narrow(const cplx* in, cplxf* out, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = cplxf{(float)in[i].x, (float)in[i].y};
}

// out (+)= the sum of the chunks' slabs in chunk order, one CTA per target
__global__ void k_translate_sum(TransArgs a, int chunks) {
    const int t = a.tbase + blockIdx.x;
    const int P2 = 2 * a.tgt.p[t] * (a.tgt.p[t] + 2);
    cplx* out = a.out + a.tgt.off[t];
    const size_t cs = (size_t)gridDim.x * a.slab_ld;   // stride between a target's chunks
    for (int e = threadIdx.x; e < P2; e += blockDim.x) {
        const cplx* q = a.slab + (size_t)blockIdx.x * a.slab_ld + e;
        cplx v = a.add ? out[e] : mk(0, 0);
        int c = 0;
        for (; c + 4 <= chunks; c += 4) {   // four loads in flight, added in chunk order
            const cplx q0 = q[c * cs], q1 = q[(c + 1) * cs], q2 = q[(c + 2) * cs], q3 = q[(c + 3) * cs];
            v = v + q0;
            v = v + q1;
            v = v + q2;
            v = v + q3;
        }
        for (; c < chunks; ++c) v = v + q[c * cs];
        out[e] = v;
    }
}

void launch_translate(const TransArgs& a, int ntargets, int chunks, cudaStream_t s) {
    if (ntargets <= 0) return;
    if (a.fp32) {
        const size_t smem = smem_bytes<cplxf>(a.pp, false);
        raise_smem_ceiling(reinterpret_cast<const void*>(k_translate<cplxf>), smem);
        k_translate<cplxf><<<dim3(ntargets, chunks), kThreads, smem, s>>>(a);
    } else {
        const size_t smem = smem_bytes<cplx>(a.pp, false);
        raise_smem_ceiling(reinterpret_cast<const void*>(k_translate<cplx>), smem);
        k_translate<cplx><<<dim3(ntargets, chunks), kThreads, smem, s>>>(a);
    }
    if (chunks > 1) k_translate_sum<<<ntargets, 256, 0, s>>>(a, chunks);
}

// ---------------------------------------------------------------------------------------------
// Several right-hand sides per CTA (the incidence directions and polarisations of one scene).
//
// The same seven stages as k_direct, each over (item, right-hand side) units with the right-hand
// side fastest: the R lanes that share an item read its d(pi/2) entries, phases and coaxial
// coefficients S(k; n, mu) once per warp instruction (one broadcast) and R consecutive values of
// the shared buffers, which hold R values per entry; one set of barriers serves R translations,
// and a thread's registers are those of the single-vector kernel.
// One CTA owns one target sphere and one tile of R right-hand sides and walks all sources of a
// bucket in order; at the end it adds T (a_n, b_n) times its sum onto y.  Launches of one
// operator application run in order on one stream and each (target, tile) belongs to one CTA, so
// the result is deterministic.
namespace {

template <class C, int R>
__host__ __device__ inline size_t smem_bytes_block(int pp, bool tabs) {
    size_t c = ((size_t)szA(pp) + szB(pp) + szAcc(pp)) * R + 4 * (size_t)(pp + 1) + (tabs ? 0 : szZ(pp));
    size_t d = (tabs ? 0 : 4 * (size_t)szZ(pp)) + 2;
    return c * sizeof(C) + d * sizeof(double) + (size_t)szNK(pp) * sizeof(short2);
}

template <class C, int R>
__device__ inline Bufs<C> carve_block(double* base, int pp, bool tabs) {
    Bufs<C> s;
    C* c = reinterpret_cast<C*>(base);
    s.A = c;           c += (size_t)szA(pp) * R;
    s.B = c;           c += (size_t)szB(pp) * R;
    s.acc = c;         c += (size_t)szAcc(pp) * R;
    s.eps = c;         c += 2 * (pp + 1);
    s.eth = c;         c += 2 * (pp + 1);
    s.zeta = c;        c += tabs ? 0 : szZ(pp);
    double* d = reinterpret_cast<double*>(c);
    s.jb = d;          d += tabs ? 0 : 2 * szZ(pp);
    s.yb = d;          d += tabs ? 0 : 2 * szZ(pp);
    s.rho = d;         d += 2;
    s.nk = reinterpret_cast<short2*>(d);
    return s;
}

// E = sum over even a, O = sum over odd a of Q[a (j+1) + o] u[a R], for both parts: delta_sum
// over one right-hand side of a buffer that holds R values per entry
template <class C, int R>
__device__ __forceinline__ void delta_sum_r(const real_of<C>* __restrict__ Q, int j, int o, int amax, const C* ua,
                                            const C* ub, C& Ea, C& Oa, C& Eb, C& Ob) {
    if constexpr (sizeof(C) == 8) {
        delta_sum_f2<R>(Q, j, o, amax, ua, ub, Ea, Oa, Eb, Ob);
        return;
    }
    using Rl = real_of<C>;
    Rl eax = 0, eay = 0, oax = 0, oay = 0, ebx = 0, eby = 0, obx = 0, oby = 0;
    const int st = j + 1;
    int a = 0;
    for (; a + 1 <= amax; a += 2) {
        const Rl q0 = __ldg(Q + a * st + o);
        const Rl q1 = __ldg(Q + (a + 1) * st + o);
        const C u0 = ua[a * R], u1 = ua[(a + 1) * R], v0 = ub[a * R], v1 = ub[(a + 1) * R];
        eax = fma(q0, u0.x, eax);
        eay = fma(q0, u0.y, eay);
        oax = fma(q1, u1.x, oax);
        oay = fma(q1, u1.y, oay);
        ebx = fma(q0, v0.x, ebx);
        eby = fma(q0, v0.y, eby);
        obx = fma(q1, v1.x, obx);
        oby = fma(q1, v1.y, oby);
    }
    if (a <= amax) {
        const Rl q0 = __ldg(Q + a * st + o);
        const C u0 = ua[a * R], v0 = ub[a * R];
        eax = fma(q0, u0.x, eax);
        eay = fma(q0, u0.y, eay);
        ebx = fma(q0, v0.x, ebx);
        eby = fma(q0, v0.y, eby);
    }
    Ea = C{eax, eay};
    Oa = C{oax, oay};
    Eb = C{ebx, eby};
    Ob = C{obx, oby};
}

// stages 2 and 6 for right-hand side r of the block layout (fwd_item with stride R)
template <class C, int R>
__device__ __forceinline__ void fwd_item_r(const real_of<C>* delta, const C* src, C* dst, int SP, int j, int s_,
                                           int amax, C eth, int r) {
    const int fold = ((j + s_) & 1) ? j + 1 : 0;
    const C* ua = src + (size_t)(off2(j) + fold) * R + r;
    C Ea, Oa, Eb, Ob;
    delta_sum_r<C, R>(delta + qoff(j), j, s_, amax, ua, ua + (size_t)SP * R, Ea, Oa, Eb, Ob);
    const real_of<C> pj_ = sgn(j), ps = sgn(s_);
    C* d = dst + (size_t)off2(j) * R + r;
#pragma unroll
    for (int part = 0; part < 2; ++part) {
        C* dp = d + (size_t)part * SP * R;
        const C E = part ? Eb : Ea, O = part ? Ob : Oa;
        const C wp = eth * (E + O);
        if (s_ == 0) {
            dp[0] = wp;
            dp[(j + 1) * R] = wp;
        } else {
            const C wm = conjg(eth) * (pj_ * (E - O));
            dp[s_ * R] = ps * (wp + wm);
            dp[(j + 1 + s_) * R] = ps * (wp - wm);
        }
    }
}

// One translation (target degree pj <- source degree pl) for the R vectors xl + r ld (r < rc),
// added into c.s.acc.  The stages of run_pair, each over (item, right-hand side) units with the
// right-hand side fastest: the R lanes of one item share its d(pi/2) entries, phases and coaxial
// coefficients and read R consecutive values of each buffer.
template <class C, int R, class Next>
__device__ inline void run_pair_block(const PairCtx<C>& c, int tid, int pj, int pl, const cplx* __restrict__ xl,
                                      int64_t ld, int rc, const C* pair_s, int cur, Next next) {
    using Rl = real_of<C>;
    using V2 = typename Vec2T<C>::type;
    const Bufs<C>& s = c.s;
    const Rl* delta = c.delta;
    const int pp = c.pp, SP = c.SP, XP = c.XP;
    const bool tabs = c.tabs;
    const int Pj = pj * (pj + 2);
    const int Pl = pl * (pl + 2);
    if (s.rho[cur] == 0.0) {
        const int pm = min(pj, pl), Pm = pm * (pm + 2);
        for (int u = tid; u < 2 * Pm * R; u += kThreads) {
            const int t = u / R, r = u % R;
            const int part = t >= Pm, e = t - part * Pm;
            if (r < rc) {
                const cplx v = xl[(size_t)r * ld + part * Pl + e];
                C& a = s.acc[(size_t)(part * Pj + e) * R + r];
                a = a + cm<C>(v.x, v.y);
            }
        }
        next(tid);
        __syncthreads();
        return;
    }
    const int kmax = min(pj, pl);
    const C* eps = s.eps + cur * (pp + 1);
    const C* eth = s.eth + cur * (pp + 1);
    // ---- 1. u = e^{i mu (phi + pi/2)} x, folded ------------------------------------------
    {
        const int items = pl * (pl + 3) / 2;
        for (int u = tid; u < items * R; u += kThreads) {
            const int t = u / R, r = u % R;
            const short2 d_ = s.nk[t];
            const int nu = d_.x, mu = d_.y;
            const int base = nu * nu - 1 + nu;
            const C e = eps[mu];
            C* U = s.A + (size_t)(off2(nu) + mu) * R + r;
            C* UB = U + (size_t)SP * R;
            double2 ap{0, 0}, am{0, 0}, bp{0, 0}, bm{0, 0};
            if (r < rc) {
                const double2* xv = reinterpret_cast<const double2*>(xl + (size_t)r * ld + base);
                ap = __ldcg(xv + mu);
                am = __ldcg(xv - mu);
                bp = __ldcg(xv + Pl + mu);
                bm = __ldcg(xv + Pl - mu);
            }
            const C ua = e * cm<C>(ap.x, ap.y), ub = e * cm<C>(bp.x, bp.y);
            if (mu == 0) {
                U[0] = ua;
                U[(nu + 1) * R] = ua;
                UB[0] = ub;
                UB[(nu + 1) * R] = ub;
            } else {
                const C va = conjg(e) * cm<C>(am.x, am.y), vb = conjg(e) * cm<C>(bm.x, bm.y);
                U[0] = ua + va;
                U[(nu + 1) * R] = ua - va;
                UB[0] = ub + vb;
                UB[(nu + 1) * R] = ub - vb;
            }
        }
        if (!tabs) {
            const int P = pj + pl + 1;
            const double* jb = s.jb + cur * szZ(pp);
            const double* yb = s.yb + cur * szZ(pp);
            for (int p = tid; p <= P; p += kThreads) {
                const cplx z = zeta_of(c.z, p, jb, yb);
                s.zeta[p] = cm<C>(z.x, z.y);
            }
        }
    }
    __syncthreads();
    // ---- 2. Delta u, e^{-i s theta} ----------------------------------------------------------
    {
        const int items = pl * (pl + 3) / 2;
        for (int b_ = 0; b_ < items * R; b_ += kThreads) {
            const int u = snake(b_, tid);
            if (u >= items * R) continue;
            const int t = u / R, r = u % R;
            const short2 d_ = s.nk[t];
            fwd_item_r<C, R>(delta, s.A, s.B, SP, d_.x, d_.y, d_.x, eth[d_.y], r);
        }
    }
    __syncthreads();
    // ---- 3. Delta^T: x'(nu, +-k) = i^{+-k} T_{+-k}, stored times (2nu+1) ------------------
    {
        const int items = pl * (pl + 3) / 2;
        for (int b_ = 0; b_ < items * R; b_ += kThreads) {
            const int u = snake(b_, tid);
            if (u >= items * R) continue;
            const int t = u / R, r = u % R;
            const short2 d_ = s.nk[t];
            const int nu = d_.x, k = d_.y;
            const int fold = ((nu + k) & 1) ? nu + 1 : 0;
            const C* va = s.B + (size_t)(off2(nu) + fold) * R + r;
            C Ea, Oa, Eb, Ob;
            delta_sum_r<C, R>(delta + qoff(nu), nu, k, nu, va, va + (size_t)SP * R, Ea, Oa, Eb, Ob);
            const Rl f = 2.0 * nu + 1.0;
            const Rl pn = sgn(nu);
            C* X = s.A + (size_t)(nu * nu - 1 + nu) * R + r;
#pragma unroll
            for (int part = 0; part < 2; ++part) {
                C* Xp = X + (size_t)part * XP * R;
                const C E = part ? Eb : Ea, O = part ? Ob : Oa;
                Xp[k * R] = ipow_mul(k, f * (E + O));
                if (k > 0) Xp[-k * R] = ipow_mul(-k, (f * pn) * (E - O));
            }
        }
    }
    __syncthreads();
    // ---- 4. w(k, mu) for a', b' at +k and -k ---------------------------------------------
    const int NW = (kmax + 1) * (pl + 2) - kmax * (kmax + 1) / 2;   // w plane stride (entries)
    {
        const double x = s.rho[cur];
        const int W = c.dt.K + 1;
        for (int u = tid; u < NW * R; u += kThreads) {
            const int t = u / R, r = u % R;
            int k = 0, rem = t;
            while (rem >= pl + 2 - k) {
                rem -= pl + 2 - k;
                ++k;
            }
            const int mu = k + rem;
            const int lo = max(1, k);
            const Rl c0 = 2.0 * mu * (mu + 1.0);
            const Rl c1m = (mu - 1 >= lo) ? x * 2.0 * (mu - 1) * c.dt.rs[mu * W + k] / (2.0 * mu - 1.0) : 0.0;
            const Rl c2p = (mu + 1 <= pl) ? x * 2.0 * (mu + 2) * c.dt.rs[(mu + 1) * W + k] / (2.0 * mu + 3.0) : 0.0;
            const Rl bk2 = 2.0 * k * x;
#pragma unroll
            for (int sg = 0; sg < 2; ++sg) {
                const int kk = sg ? -k : k;
                const Rl bs = sg ? -bk2 : bk2;
                C av[3], bv[3];
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    const int nu = mu - 1 + d;
                    const bool ok = nu >= lo && nu <= pl;
                    const int o = nu * nu - 1 + nu + kk;
                    av[d] = ok ? s.A[(size_t)o * R + r] : C{0, 0};
                    bv[d] = ok ? s.A[(size_t)(XP + o) * R + r] : C{0, 0};
                }
                const C ia = bs * bv[1] + c1m * av[0] - c2p * av[2];
                const C ib = bs * av[1] + c1m * bv[0] - c2p * bv[2];
                s.B[((size_t)(2 * sg) * NW + t) * R + r] = C{c0 * av[1].x - ia.y, c0 * av[1].y + ia.x};
                s.B[((size_t)(2 * sg + 1) * NW + t) * R + r] = C{c0 * bv[1].x - ib.y, c0 * bv[1].y + ib.x};
            }
        }
    }
    __syncthreads();
    // ---- 5. out(k, n) = sum_mu S(k; n, mu) w(k, mu), folded for the back rotation ----------
    {
        const int rows_tot = pj + (kmax >= 1 ? kmax * pj - (kmax - 1) * kmax / 2 : 0);
        const int M2 = max(pj, pl) + 2;
        for (int b_ = 0; b_ < rows_tot * R; b_ += kThreads) {
            const int u = snake(b_, tid);
            if (u >= rows_tot * R) continue;
            const int t = u / R, r = u % R;
            int k = 0, rem = t;
            for (;;) {
                const int rk = pj - max(1, k) + 1;
                if (rem < rk) break;
                rem -= rk;
                ++k;
            }
            const int n = max(1, k) + rem;
            const C* w = s.B + (size_t)(k * (pl + 2) - k * (k - 1) / 2) * R + r;
            const size_t NWR = (size_t)NW * R;
            const int cnt = pl + 2 - k;
            Mac4<C> acc;
            if (tabs) {
                const int Wk = M2 - k;
                const V2* sp = reinterpret_cast<const V2*>(pair_s + pair_block_offset(k, M2, M2) + (n - k));
                int q = 0;
                for (; q + kPrefetch5 <= cnt; q += kPrefetch5) {
                    V2 sv[kPrefetch5];
#pragma unroll
                    for (int v = 0; v < kPrefetch5; ++v) sv[v] = __ldcg(sp + (q + v) * Wk);
#pragma unroll
                    for (int v = 0; v < kPrefetch5; ++v) {
                        const size_t o = (size_t)(q + v) * R;
                        acc.add(C{sv[v].x, sv[v].y}, w[o], w[NWR + o], w[2 * NWR + o], w[3 * NWR + o]);
                    }
                }
                for (; q < cnt; ++q) {
                    const V2 sv = __ldcg(sp + q * Wk);
                    const size_t o = (size_t)q * R;
                    acc.add(C{sv.x, sv.y}, w[o], w[NWR + o], w[2 * NWR + o], w[3 * NWR + o]);
                }
            } else {
                const int Wg = c.g.NM - k + 1;
                const size_t plane = (size_t)Wg * Wg;
                const double* G = c.g.gs + c.g.koff[k] + (n - k);
                for (int q = 0; q < cnt; ++q) {
                    const int mu = k + q;
                    const double* gp = G + (size_t)(mu - k) * Wg;
                    const int qm = min(n, mu);
                    int p = n + mu;
                    double sx = 0.0, sy = 0.0;
                    for (int qq = 0; qq <= qm; ++qq, p -= 2) {
                        const double gq = __ldg(gp + qq * plane);
                        sx += gq * s.zeta[p].x;
                        sy += gq * s.zeta[p].y;
                    }
                    const size_t o = (size_t)q * R;
                    acc.add(cm<C>(sx, sy), w[o], w[NWR + o], w[2 * NWR + o], w[3 * NWR + o]);
                }
            }
            const Rl f = sgn(k) / (2.0 * n * (n + 1.0));
            C* U = s.A + (size_t)(off2(n) + k) * R + r;
            C* UB = U + (size_t)SP * R;
            if (k == 0) {
                const C a0 = f * acc.get(0), b0 = f * acc.get(1);
                U[0] = a0;
                U[(n + 1) * R] = a0;
                UB[0] = b0;
                UB[(n + 1) * R] = b0;
            } else {
                const C ap = ipow_mul(-k, f * acc.get(0)), am = ipow_mul(k, f * acc.get(2));
                const C bp = ipow_mul(-k, f * acc.get(1)), bm = ipow_mul(k, f * acc.get(3));
                U[0] = ap + am;
                U[(n + 1) * R] = ap - am;
                UB[0] = bp + bm;
                UB[(n + 1) * R] = bp - bm;
            }
        }
    }
    __syncthreads();
    // ---- 6. Delta on the translated field, e^{-i s theta} (orders |k| <= kmax only) ----------
    {
        const int items = pj * (pj + 3) / 2;
        for (int b_ = 0; b_ < items * R; b_ += kThreads) {
            const int u = snake(b_, tid);
            if (u >= items * R) continue;
            const int t = u / R, r = u % R;
            const short2 d_ = s.nk[t];
            fwd_item_r<C, R>(delta, s.A, s.B, SP, d_.x, d_.y, min((int)d_.x, kmax), eth[d_.y], r);
        }
    }
    __syncthreads();
    // ---- 7. Delta^T, phase, accumulate; then the next pair's tables ---------------------------
    {
        const int items = pj * (pj + 3) / 2;
        for (int b_ = 0; b_ < items * R; b_ += kThreads) {
            const int u = snake(b_, tid);
            if (u >= items * R) continue;
            const int t = u / R, r = u % R;
            const short2 d_ = s.nk[t];
            const int n = d_.x, m = d_.y;
            const int fold = ((n + m) & 1) ? n + 1 : 0;
            const C* va = s.B + (size_t)(off2(n) + fold) * R + r;
            C Ea, Oa, Eb, Ob;
            delta_sum_r<C, R>(delta + qoff(n), n, m, n, va, va + (size_t)SP * R, Ea, Oa, Eb, Ob);
            const Rl pn = sgn(n);
            const C e = eps[m];
            const int base = n * n - 1 + n;
#pragma unroll
            for (int part = 0; part < 2; ++part) {
                const C E = part ? Eb : Ea, O = part ? Ob : Oa;
                C& ap = s.acc[(size_t)(part * Pj + base + m) * R + r];
                ap = ap + conjg(e) * (E + O);
                if (m > 0) {
                    C& am = s.acc[(size_t)(part * Pj + base - m) * R + r];
                    am = am + e * (pn * (E - O));
                }
            }
        }
        next(tid);
    }
    __syncthreads();
}

}  // namespace

// CTAs per SM the block kernel's registers are set for (the single-vector operator's bounds:
// its per-thread work is the same)
template <class C, int R>
__global__ void __launch_bounds__(kThreads, DirectOcc<C>::ctas) k_direct_block(BlockArgs ba, DirectBucket bk) {
    extern __shared__ __align__(16) double smem_d[];
    const DirectArgs& a = ba.d;
    const SceneView& sc = a.sc;
    const int pp = bk.pp;
    const C* stab = stab_of(a, (C*)nullptr);
    const bool tabs = stab != nullptr;
    const Bufs<C> s = carve_block<C, R>(smem_d, pp, tabs);
    const int tile = blockIdx.x;
    const int j = bk.targets[blockIdx.y];
    if (!sc.couple[j]) return;
    const int r0 = tile * R;
    const int rc = min(R, ba.nrhs - r0);
    const int tid = threadIdx.x;
    const int pj = sc.p[j];
    const int Pj = pj * (pj + 2);
    const int SP = pp * (pp + 3);
    const int XP = pp * (pp + 2);
    const PairCtx<C> ctx{s, delta_of(a, (C*)nullptr), a.dt, a.g, a.z, pp, SP, XP, tabs};
    for (int t = tid; t < 2 * Pj * R; t += kThreads) s.acc[t] = C{0, 0};
    for (int t = tid; t < pp * (pp + 3) / 2; t += kThreads) {
        int n, k;
        decode_nk(t, n, k);
        s.nk[t] = make_short2((short)n, (short)k);
    }
    auto block = [&](int l) -> const C* {
        return tabs ? stab + a.pt.pair_off[pair_index(min(j, l), max(j, l), sc.n)] : nullptr;
    };
    auto disp = [&](int l) {
        return Disp{sc.centres + 3 * (size_t)j, sc.centres + 3 * (size_t)l, sc.k, 1.0, {0.0, 0.0, 0.0}};
    };
    const cplx* X = ba.x + (size_t)r0 * ba.ld;
    int i = 0;
    if (i < bk.nsources && bk.sources[i] == j) ++i;
    if (i < bk.nsources) {
        const int l = bk.sources[i];
        prep_pair(s, disp(l), a.z, block(l), pj, sc.p[l], pp, 0, tid, !tabs);
    }
    __syncthreads();
    int cur = 0;
    while (i < bk.nsources) {
        const int l = bk.sources[i];
        int inext = i + 1;
        if (inext < bk.nsources && bk.sources[inext] == j) ++inext;
        run_pair_block<C, R>(ctx, tid, pj, sc.p[l], X + sc.off[l], ba.ld, rc, block(l), cur, [&](int t) {
            if (inext < bk.nsources) {
                const int ln = bk.sources[inext];
                prep_pair(s, disp(ln), a.z, block(ln), pj, sc.p[ln], pp, cur ^ 1, t, !tabs);
            }
        });
        cur ^= 1;
        i = inext;
    }
    // y += T sum, T = diag(a_n, b_n) of the target
    cplx* Y = ba.y + (size_t)r0 * ba.ld + sc.off[j];
    for (int u = tid; u < 2 * Pj * R; u += kThreads) {
        const int r = u / (2 * Pj), t = u - r * 2 * Pj;   // right-hand side slowest: coalesced rows of y
        if (r >= rc) continue;
        const int tt = t < Pj ? t : t - Pj;
        int n, m;
        decode_nm(tt, n, m);
        const cplx tm = (t < Pj) ? sc.an[(size_t)j * sc.pmax + n - 1] : sc.bn[(size_t)j * sc.pmax + n - 1];
        const C av = s.acc[(size_t)t * R + r];
        cplx* yp = Y + (size_t)r * ba.ld + t;
        *yp = *yp + tm * mk(av.x, av.y);
    }
}

size_t block_smem_bytes(int pp, bool tabs, bool fp32, int R) {
    if (fp32) {
        switch (R) {
            case 1: return smem_bytes_block<cplxf, 1>(pp, tabs);
            case 2: return smem_bytes_block<cplxf, 2>(pp, tabs);
            case 4: return smem_bytes_block<cplxf, 4>(pp, tabs);
            case 8: return smem_bytes_block<cplxf, 8>(pp, tabs);
            case 16: return smem_bytes_block<cplxf, 16>(pp, tabs);
        }
    } else {
        switch (R) {
            case 1: return smem_bytes_block<cplx, 1>(pp, tabs);
            case 2: return smem_bytes_block<cplx, 2>(pp, tabs);
            case 4: return smem_bytes_block<cplx, 4>(pp, tabs);
            case 8: return smem_bytes_block<cplx, 8>(pp, tabs);
        }
    }
    return 0;
}

template <class C, int R>
static void launch_block_t(const BlockArgs& a, const DirectBucket& b, cudaStream_t s) {
    const bool tabs = stab_of_host<C>(a.d) != nullptr;
    const size_t smem = smem_bytes_block<C, R>(b.pp, tabs);
    raise_smem_ceiling(reinterpret_cast<const void*>(k_direct_block<C, R>), smem);
    dim3 grid((a.nrhs + R - 1) / R, b.ntargets);
    k_direct_block<C, R><<<grid, kThreads, smem, s>>>(a, b);
}

bool launch_direct_block(const BlockArgs& a, const DirectBucket& b, int R, cudaStream_t s) {
    if (a.d.fp32) {
        switch (R) {
            case 1: launch_block_t<cplxf, 1>(a, b, s); return true;
            case 2: launch_block_t<cplxf, 2>(a, b, s); return true;
            case 4: launch_block_t<cplxf, 4>(a, b, s); return true;
            case 8: launch_block_t<cplxf, 8>(a, b, s); return true;
            case 16: launch_block_t<cplxf, 16>(a, b, s); return true;
        }
    } else {
        switch (R) {
            case 1: launch_block_t<cplx, 1>(a, b, s); return true;
            case 2: launch_block_t<cplx, 2>(a, b, s); return true;
            case 4: launch_block_t<cplx, 4>(a, b, s); return true;
            case 8: launch_block_t<cplx, 8>(a, b, s); return true;
        }
    }
    return false;
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

}  // namespace foggy
