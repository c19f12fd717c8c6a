// Krylov-space kernels of the device GMRES (replacing the CERFACS drive_zgmres loop the
// reference runs on the host, FoggySim/src/lib/mie_theory/lib_solver_GMRES.f90:116-316).
// All reductions are two-pass with a fixed order, so a solve is bit-reproducible.
#include "foggy_kernels.cuh"

namespace foggy {

namespace {
constexpr int kT = 256;
constexpr int kMaxDots = 64;   // Krylov vectors handled per dots launch
}

// conj(v) . w over [lo, hi) by one warp: lanes stride the slice, then a fixed butterfly of shuffles
__device__ __forceinline__ cplx warp_dot(const cplx* __restrict__ v, const cplx* __restrict__ w, int64_t lo, int64_t hi,
                                         int lane) {
    double sx = 0.0, sy = 0.0;
    for (int64_t t = lo + lane; t < hi; t += 32) {
        const cplx a = v[t], b = w[t];
        sx += a.x * b.x + a.y * b.y;
        sy += a.x * b.y - a.y * b.x;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sx += __shfl_xor_sync(0xffffffffu, sx, o);
        sy += __shfl_xor_sync(0xffffffffu, sy, o);
    }
    return mk(sx, sy);
}

// part[i * kRedBlocks + block] = partial sum of conj(V_i) . w over the block's slice; warp q of the
// block takes the vectors i = q, q + 8, ... (no block-wide barrier per vector)
__global__ void __launch_bounds__(kT) k_dots_partial(const cplx* V, int64_t ld, int nv, const cplx* w, int64_t n,
                                                     cplx* part) {
    const int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
    const int64_t lo = (int64_t)blockIdx.x * chunk;
    const int64_t hi = min(n, lo + chunk);
    const int lane = threadIdx.x & 31, q = threadIdx.x >> 5;
    for (int i = q; i < nv; i += kT / 32) {
        const cplx d = warp_dot(V + (size_t)i * ld, w, lo, hi, lane);
        if (lane == 0) part[(size_t)i * gridDim.x + blockIdx.x] = d;
    }
}

// out[i] (+)= sum over blocks of part[i], one block per i
__global__ void __launch_bounds__(kT) k_dots_reduce(const cplx* part, int nv, cplx* out, int accumulate) {
    __shared__ double red_x[kT], red_y[kT];
    int i = blockIdx.x;
    double sx = 0.0, sy = 0.0;
    for (int b = threadIdx.x; b < kRedBlocks; b += blockDim.x) {
        sx += part[(size_t)i * kRedBlocks + b].x;
        sy += part[(size_t)i * kRedBlocks + b].y;
    }
    red_x[threadIdx.x] = sx;
    red_y[threadIdx.x] = sy;
    __syncthreads();
    for (int s = kT / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            red_x[threadIdx.x] += red_x[threadIdx.x + s];
            red_y[threadIdx.x] += red_y[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        cplx v = mk(red_x[0], red_y[0]);
        out[i] = accumulate ? out[i] + v : v;
    }
}

// w -= sum_i h_i V_i
__global__ void k_axpy_multi(const cplx* V, int64_t ld, int nv, const cplx* h, cplx* w, int64_t n) {
    __shared__ cplx hs[kMaxDots];
    for (int i = threadIdx.x; i < nv; i += blockDim.x) hs[i] = h[i];
    __syncthreads();
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        cplx acc = w[t];
        for (int i = 0; i < nv; ++i) acc = acc - hs[i] * V[(size_t)i * ld + t];
        w[t] = acc;
    }
}

__global__ void __launch_bounds__(kT) k_norm_partial(const cplx* w, int64_t n, double* part) {
    __shared__ double red[kT];
    int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
    int64_t lo = (int64_t)blockIdx.x * chunk;
    int64_t hi = min(n, lo + chunk);
    double s = 0.0;
    for (int64_t t = lo + threadIdx.x; t < hi; t += blockDim.x) s += w[t].x * w[t].x + w[t].y * w[t].y;
    red[threadIdx.x] = s;
    __syncthreads();
    for (int k = kT / 2; k > 0; k >>= 1) {
        if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void __launch_bounds__(kT) k_norm_reduce(const double* part, double* out) {
    __shared__ double red[kT];
    double s = 0.0;
    for (int b = threadIdx.x; b < kRedBlocks; b += blockDim.x) s += part[b];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int k = kT / 2; k > 0; k >>= 1) {
        if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = sqrt(red[0]);
}

// v = w / nrm (v = 0 when nrm == 0)
__global__ void k_scale_copy(const cplx* w, const double* nrm, cplx* v, int64_t n) {
    double r = nrm[0];
    double inv = (r != 0.0) ? 1.0 / r : 0.0;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        v[t] = inv * w[t];
}

__global__ void k_sub(const cplx* b, const cplx* ax, cplx* r, int64_t n) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        r[t] = b[t] - ax[t];
}

// g = (beta, 0, ...) at the start of a restart cycle
__global__ void k_init_cycle(cplx* g, int m1, const double* beta, int* flags) {
    for (int i = threadIdx.x; i < m1; i += blockDim.x) g[i] = mk(0, 0);
    __syncthreads();
    if (threadIdx.x == 0) {
        g[0] = mk(beta[0], 0.0);
        flags[0] = 0;
    }
}

// Column k of the Hessenberg matrix: H[0..k][k] = h + c (both Gram-Schmidt passes), H[k+1][k] = hn.  Applies the previous
// Givens rotations, forms the new one, updates g and writes |g[k+1]| to res_est.
// H is row-major with leading dimension ldh (= restart).
__global__ void k_givens(cplx* H, int ldh, cplx* cs, double* sn, cplx* g, const cplx* h, const cplx* c,
                         const double* hn, int k, double* res_est, int* flags) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int i = 0; i <= k; ++i) H[(size_t)i * ldh + k] = h[i] + c[i];
    double hk1 = hn[0];
    for (int i = 0; i < k; ++i) {
        cplx a = H[(size_t)i * ldh + k], b = H[(size_t)(i + 1) * ldh + k];
        H[(size_t)i * ldh + k] = conjg(cs[i]) * a + sn[i] * b;
        H[(size_t)(i + 1) * ldh + k] = mk(-sn[i], 0) * a + cs[i] * b;
    }
    cplx a = H[(size_t)k * ldh + k];
    double den = sqrt(a.x * a.x + a.y * a.y + hk1 * hk1);
    if (den == 0.0) {
        flags[0] = 1;   // breakdown
        res_est[0] = 0.0;
        return;
    }
    cs[k] = mk(a.x / den, a.y / den);
    sn[k] = hk1 / den;
    H[(size_t)k * ldh + k] = mk(den, 0);
    cplx gk = g[k];
    g[k + 1] = mk(-sn[k], 0) * gk;
    g[k] = conjg(cs[k]) * gk;
    res_est[0] = sqrt(g[k + 1].x * g[k + 1].x + g[k + 1].y * g[k + 1].y);
    if (!isfinite(res_est[0])) flags[0] = 2;
}

// back substitution H[0:k,0:k] y = g[0:k]
__global__ void k_trisolve(const cplx* H, int ldh, const cplx* g, int k, cplx* y) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int i = k - 1; i >= 0; --i) {
        cplx s = g[i];
        for (int t = i + 1; t < k; ++t) s = s - H[(size_t)i * ldh + t] * y[t];
        y[i] = cdiv(s, H[(size_t)i * ldh + i]);
    }
}

// x += sum_{i<k} y_i V_i
__global__ void k_update_x(cplx* x, const cplx* V, int64_t ld, const cplx* y, int k, int64_t n) {
    __shared__ cplx ys[kMaxDots];
    for (int i = threadIdx.x; i < k; i += blockDim.x) ys[i] = y[i];
    __syncthreads();
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        cplx acc = x[t];
        for (int i = 0; i < k; ++i) acc = acc + ys[i] * V[(size_t)i * ld + t];
        x[t] = acc;
    }
}


// ---- several right-hand sides ----------------------------------------------------------------
// One Krylov space per right-hand side, advanced in lock step so that the operator is applied to
// the whole block.  Slot b (blockIdx.y) owns basis vector i at V + i ldi + b ld; slots whose
// live[b] is 0 have left the current restart cycle and are skipped.  The same two-pass
// fixed-order reductions as above, so each slot's arithmetic does not depend on the others.

// part[(b nv + i) kRedBlocks + block] = partial sum of conj(V_i) . w_b
__global__ void __launch_bounds__(kT) k_dots_partial_b(const cplx* V, int64_t ldi, int64_t ld, int nv,
                                                       const cplx* W, int64_t n, const int* live, cplx* part) {
    const int b = blockIdx.y;
    if (!live[b]) return;
    const cplx* w = W + (size_t)b * ld;
    const int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
    const int64_t lo = (int64_t)blockIdx.x * chunk;
    const int64_t hi = min(n, lo + chunk);
    const int lane = threadIdx.x & 31, q = threadIdx.x >> 5;
    for (int i = q; i < nv; i += kT / 32) {
        const cplx d = warp_dot(V + (size_t)i * ldi + (size_t)b * ld, w, lo, hi, lane);
        if (lane == 0) part[((size_t)b * nv + i) * gridDim.x + blockIdx.x] = d;
    }
}

// out[b ostride + i] = sum over blocks of part[b][i]; grid (nv, slots)
__global__ void __launch_bounds__(kT) k_dots_reduce_b(const cplx* part, int nv, const int* live, cplx* out,
                                                      int ostride) {
    __shared__ double red_x[kT], red_y[kT];
    const int i = blockIdx.x, b = blockIdx.y;
    if (!live[b]) return;
    const cplx* p = part + ((size_t)b * nv + i) * kRedBlocks;
    double sx = 0.0, sy = 0.0;
    for (int q = threadIdx.x; q < kRedBlocks; q += blockDim.x) {
        sx += p[q].x;
        sy += p[q].y;
    }
    red_x[threadIdx.x] = sx;
    red_y[threadIdx.x] = sy;
    __syncthreads();
    for (int s = kT / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            red_x[threadIdx.x] += red_x[threadIdx.x + s];
            red_y[threadIdx.x] += red_y[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) out[(size_t)b * ostride + i] = mk(red_x[0], red_y[0]);
}

// w_b -= sum_i h[b hstride + i] V_i(b)
__global__ void k_axpy_multi_b(const cplx* V, int64_t ldi, int64_t ld, int nv, const cplx* h, int hstride,
                               cplx* W, int64_t n, const int* live) {
    __shared__ cplx hs[kMaxDots];
    const int b = blockIdx.y;
    if (!live[b]) return;
    for (int i = threadIdx.x; i < nv; i += blockDim.x) hs[i] = h[(size_t)b * hstride + i];
    __syncthreads();
    cplx* w = W + (size_t)b * ld;
    const cplx* Vb = V + (size_t)b * ld;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        cplx acc = w[t];
        for (int i = 0; i < nv; ++i) acc = acc - hs[i] * Vb[(size_t)i * ldi + t];
        w[t] = acc;
    }
}

// nrm[b nstride] = ||w_b||; grid (kRedBlocks, slots) then (1, slots)
__global__ void __launch_bounds__(kT) k_norm_partial_b(const cplx* W, int64_t ld, int64_t n, const int* live,
                                                       double* part) {
    __shared__ double red[kT];
    const int b = blockIdx.y;
    if (live && !live[b]) return;
    const cplx* w = W + (size_t)b * ld;
    int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
    int64_t lo = (int64_t)blockIdx.x * chunk;
    int64_t hi = min(n, lo + chunk);
    double s = 0.0;
    for (int64_t t = lo + threadIdx.x; t < hi; t += blockDim.x) s += w[t].x * w[t].x + w[t].y * w[t].y;
    red[threadIdx.x] = s;
    __syncthreads();
    for (int k = kT / 2; k > 0; k >>= 1) {
        if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[(size_t)b * gridDim.x + blockIdx.x] = red[0];
}

__global__ void __launch_bounds__(kT) k_norm_reduce_b(const double* part, const int* live, double* out,
                                                      int ostride) {
    __shared__ double red[kT];
    const int b = blockIdx.y;
    if (live && !live[b]) return;
    double s = 0.0;
    for (int q = threadIdx.x; q < kRedBlocks; q += blockDim.x) s += part[(size_t)b * kRedBlocks + q];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int k = kT / 2; k > 0; k >>= 1) {
        if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[(size_t)b * ostride] = sqrt(red[0]);
}

// v_b = w_b / nrm[b nstride]
__global__ void k_scale_copy_b(const cplx* W, int64_t ldw, const double* nrm, int nstride, cplx* Vout, int64_t ldv,
                               int64_t n, const int* live) {
    const int b = blockIdx.y;
    if (live && !live[b]) return;
    const double r = nrm[(size_t)b * nstride];
    const double inv = (r != 0.0) ? 1.0 / r : 0.0;
    const cplx* w = W + (size_t)b * ldw;
    cplx* v = Vout + (size_t)b * ldv;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        v[t] = inv * w[t];
}

// r_b = b_b - (A x)_b
__global__ void k_sub_b(const cplx* Bv, const cplx* AX, cplx* Rv, int64_t ld, int64_t n) {
    const size_t o = (size_t)blockIdx.y * ld;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        Rv[o + t] = Bv[o + t] - AX[o + t];
}

// Start of a restart cycle for every slot: g = (beta, 0, ...), live = 1, kend = 0.
__global__ void k_init_cycle_b(cplx* g, int m1, const double* beta, int nslots, int* live, int* kend) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nslots) return;
    for (int i = 0; i < m1; ++i) g[(size_t)b * m1 + i] = mk(0, 0);
    g[(size_t)b * m1] = mk(beta[b], 0.0);
    live[b] = 1;
    kend[b] = 0;
}

// Column k of each live slot's Hessenberg matrix, its Givens rotations and residual estimate
// (k_givens per slot).  A slot leaves the cycle after this step (live = 0, kend = k + 1) when its
// estimate reaches tol_abs[b], at breakdown (kend = k, flags 1) or on a non-finite value (flags 2).
__global__ void k_givens_b(cplx* H, int m, cplx* cs, double* sn, cplx* g, const cplx* h, const cplx* c,
                           const double* hn, int k, const double* tol_abs, double* res_est, int* flags, int* live,
                           int* kend, int nslots) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nslots || !live[b]) return;
    cplx* Hb = H + (size_t)b * (m + 1) * m;
    cplx* csb = cs + (size_t)b * m;
    double* snb = sn + (size_t)b * m;
    cplx* gb = g + (size_t)b * (m + 1);
    const cplx* hb = h + (size_t)b * (m + 1);
    const cplx* cb = c + (size_t)b * (m + 1);
    for (int i = 0; i <= k; ++i) Hb[(size_t)i * m + k] = hb[i] + cb[i];
    const double hk1 = hn[b];
    for (int i = 0; i < k; ++i) {
        cplx a = Hb[(size_t)i * m + k], d = Hb[(size_t)(i + 1) * m + k];
        Hb[(size_t)i * m + k] = conjg(csb[i]) * a + snb[i] * d;
        Hb[(size_t)(i + 1) * m + k] = mk(-snb[i], 0) * a + csb[i] * d;
    }
    cplx a = Hb[(size_t)k * m + k];
    double den = sqrt(a.x * a.x + a.y * a.y + hk1 * hk1);
    if (den == 0.0) {
        flags[b] = 1;
        res_est[b] = 0.0;
        live[b] = 0;
        kend[b] = k;
        return;
    }
    csb[k] = mk(a.x / den, a.y / den);
    snb[k] = hk1 / den;
    Hb[(size_t)k * m + k] = mk(den, 0);
    cplx gk = gb[k];
    gb[k + 1] = mk(-snb[k], 0) * gk;
    gb[k] = conjg(csb[k]) * gk;
    const double re = sqrt(gb[k + 1].x * gb[k + 1].x + gb[k + 1].y * gb[k + 1].y);
    res_est[b] = re;
    kend[b] = k + 1;
    if (!isfinite(re)) {
        flags[b] = 2;
        live[b] = 0;
    } else if (re <= tol_abs[b] || hk1 == 0.0 || k + 1 == m) {
        live[b] = 0;
    }
}

// y_b = H_b^{-1} g_b over the slot's kend[b] columns, then x_b += sum_i y_i V_i(b)
__global__ void k_trisolve_b(const cplx* H, int m, const cplx* g, const int* kend, cplx* y, int nslots) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nslots) return;
    const int k = kend[b];
    const cplx* Hb = H + (size_t)b * (m + 1) * m;
    const cplx* gb = g + (size_t)b * (m + 1);
    cplx* yb = y + (size_t)b * (m + 1);
    for (int i = k - 1; i >= 0; --i) {
        cplx s = gb[i];
        for (int t = i + 1; t < k; ++t) s = s - Hb[(size_t)i * m + t] * yb[t];
        yb[i] = cdiv(s, Hb[(size_t)i * m + i]);
    }
}

__global__ void k_update_x_b(cplx* X, int64_t ld, const cplx* V, int64_t ldi, const cplx* y, int ystride,
                             const int* kend, int64_t n) {
    __shared__ cplx ys[kMaxDots];
    const int b = blockIdx.y;
    const int k = kend[b];
    if (k == 0) return;
    for (int i = threadIdx.x; i < k; i += blockDim.x) ys[i] = y[(size_t)b * ystride + i];
    __syncthreads();
    cplx* x = X + (size_t)b * ld;
    const cplx* Vb = V + (size_t)b * ld;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        cplx acc = x[t];
        for (int i = 0; i < k; ++i) acc = acc + ys[i] * Vb[(size_t)i * ldi + t];
        x[t] = acc;
    }
}

}  // namespace foggy
