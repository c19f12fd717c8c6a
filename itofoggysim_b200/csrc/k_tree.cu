// Octree keys of the sphere centres (libtree).  Bit-exact restatement of the reference's
// scaling (libtree/src/lib/lib_tree.f90:320-374) and universal index
// (libtree/src/lib/lib_tree_helper_functions.f90:202-364, 532-614, 1204-1266):
//   * coordinates are scaled by one length D = max_d (x_max,d - x_min,d)(1 + 2^-52) into [0,1);
//   * the 64 fraction bits of each scaled coordinate are read from its IEEE-754 pattern
//     (mantissa with the implicit one, shifted right by 1022 - exponent);
//   * bits are interleaved with dimension 1 (x) most significant in each 3-bit group and the
//     universal index at level l is the top 3 l bits.
// The level-21 key of one sphere is one 63-bit integer; every coarser index is a right shift.
#include "foggy_kernels.cuh"

namespace foggy {

// out[0..2] = min per dimension, out[3..5] = max; one block
__global__ void k_minmax(int n, const double* c, double* out) {
    __shared__ double smin[3][256], smax[3][256];
    for (int d = 0; d < 3; ++d) {
        double lo = c[d], hi = c[d];
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            lo = fmin(lo, c[3 * (size_t)i + d]);
            hi = fmax(hi, c[3 * (size_t)i + d]);
        }
        smin[d][threadIdx.x] = lo;
        smax[d][threadIdx.x] = hi;
    }
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int d = 0; d < 3; ++d) {
                smin[d][threadIdx.x] = fmin(smin[d][threadIdx.x], smin[d][threadIdx.x + s]);
                smax[d][threadIdx.x] = fmax(smax[d][threadIdx.x], smax[d][threadIdx.x + s]);
            }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int d = 0; d < 3; ++d) {
            out[d] = smin[d][0];
            out[3 + d] = smax[d][0];
        }
}

__device__ __forceinline__ unsigned long long coordinate_binary(double f) {
    unsigned long long bits = (unsigned long long)__double_as_longlong(f);
    long long e = (long long)(bits >> 52);
    unsigned long long mant = (bits << 11) | (1ull << 63);
    long long shift = 1023 - e - 1;
    if (shift >= 64) return 0ull;
    if (shift <= 0) return mant;
    return mant >> shift;
}

// top 21 fraction bits per dimension, interleaved x|y|z per level -> 63-bit level-21 key
__device__ __forceinline__ unsigned long long key21(double x, double y, double z) {
    unsigned long long bx = coordinate_binary(x) >> 43;
    unsigned long long by = coordinate_binary(y) >> 43;
    unsigned long long bz = coordinate_binary(z) >> 43;
    unsigned long long key = 0;
    for (int b = 20; b >= 0; --b)
        key = (key << 3) | (((bx >> b) & 1ull) << 2) | (((by >> b) & 1ull) << 1) | ((bz >> b) & 1ull);
    return key;
}

__global__ void k_morton(int n, const double* c, const double* mm, unsigned long long* key, int* idx) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double D[3];
    for (int d = 0; d < 3; ++d) D[d] = __dmul_rn(__dsub_rn(mm[3 + d], mm[d]), 1.0 + 2.220446049250313e-16);
    double Dm = fmax(D[0], fmax(D[1], D[2]));
    double s[3];
    for (int d = 0; d < 3; ++d) s[d] = (Dm > 0.0) ? __ddiv_rn(__dsub_rn(c[3 * (size_t)i + d], mm[d]), Dm) : 0.0;
    key[i] = key21(s[0], s[1], s[2]);
    idx[i] = i;
}

// level at which sorted elements i and i+s still share a box, plus one
// (lib_tree_get_level_max, libtree/src/lib/lib_tree.f90:1188-1242)
__global__ void k_level_max(int n, int s, const unsigned long long* key, int* lmax) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i + s >= n) return;
    unsigned long long x = key[i] ^ key[i + s];
    int lev;
    if (x == 0ull) {
        lev = 21;
    } else {
        int h = 63 - __clzll((long long)x);   // highest differing bit, 0..62
        lev = 21 - h / 3;
        if (h / 3 >= 21) lev = 0;
    }
    atomicMax(lmax, lev);
}

__global__ void k_uindex_points(int n, const double* pts, int l, long long* out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    unsigned long long k = key21(pts[3 * (size_t)i], pts[3 * (size_t)i + 1], pts[3 * (size_t)i + 2]);
    out[i] = (long long)(k >> (3 * (21 - l)));
}

}  // namespace foggy
