// Krylov-space kernels of the device GMRES (replacing the CERFACS drive_zgmres loop the
// reference runs on the host, FoggySim/src/lib/mie_theory/lib_solver_GMRES.f90:116-316).
// All reductions are two-pass with a fixed order, so a solve is bit-reproducible.
#include "foggy_kernels.cuh"

namespace foggy {

namespace {
constexpr int kT = 256;
constexpr int kMaxDots = 64;   // Krylov vectors handled per dots launch
}

// part[i * kRedBlocks + block] = partial sum of conj(V_i) . w over the block's slice
__global__ void __launch_bounds__(kT) k_dots_partial(const cplx* V, int64_t ld, int nv, const cplx* w, int64_t n,
                                                     cplx* part) {
    __shared__ double red_x[kT], red_y[kT];
    int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
    int64_t lo = (int64_t)blockIdx.x * chunk;
    int64_t hi = min(n, lo + chunk);
    for (int i = 0; i < nv; ++i) {
        const cplx* v = V + (size_t)i * ld;
        double sx = 0.0, sy = 0.0;
        for (int64_t t = lo + threadIdx.x; t < hi; t += blockDim.x) {
            cplx a = v[t], b = w[t];
            sx += a.x * b.x + a.y * b.y;
            sy += a.x * b.y - a.y * b.x;
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
        if (threadIdx.x == 0) part[(size_t)i * gridDim.x + blockIdx.x] = mk(red_x[0], red_y[0]);
        __syncthreads();
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

}  // namespace foggy
