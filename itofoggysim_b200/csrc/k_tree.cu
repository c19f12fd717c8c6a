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


// ---- ML-FMM hierarchy and lists on the device ------------------------------------------------
// The spheres are sorted by their level-21 key, so the spheres of any box are one contiguous run
// of the sorted order.  Boxes of levels l_min..l_max get one global id, level by level in
// ascending Morton order: flag[li n + i] = 1 where sorted sphere i starts a box at level
// l_min + li, and the inclusive scan of the flags minus one is the box of sphere i at that level
// (lib_ml_fmm_hf_create_hierarchy, libmlfmm/src/lib/lib_ml_fmm_helper_functions.f90:366-457).
__global__ void k_tree_flags(int n, int nlev, int lmin, const unsigned long long* key, int* flag) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)nlev * n) return;
    const int li = (int)(idx / n), i = (int)(idx - (int64_t)li * n);
    const int sh = 3 * (21 - (lmin + li));
    flag[idx] = (i == 0 || (key[i] >> sh) != (key[i - 1] >> sh)) ? 1 : 0;
}

__global__ void k_tree_boxes(int n, int nlev, int lmin, const unsigned long long* key, const int* incl,
                             long long* box_n, int* box_level, int* run_start, int* level_base) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)nlev * n) return;
    const int li = (int)(idx / n), i = (int)(idx - (int64_t)li * n);
    const int sh = 3 * (21 - (lmin + li));
    const int b = incl[idx] - 1;
    if (i == 0 || (key[i] >> sh) != (key[i - 1] >> sh)) {
        box_n[b] = (long long)(key[i] >> sh);
        box_level[b] = lmin + li;
        run_start[b] = i;
        if (i == 0) level_base[li] = b;
    }
    if (idx == (int64_t)nlev * n - 1) level_base[nlev] = b + 1;
}

__device__ __forceinline__ int level_of_box(int b, int nlev, const int* level_base) {
    int li = 0;
    while (li + 1 < nlev && b >= level_base[li + 1]) ++li;
    return li;
}

// run ends and parents (lib_tree_get_parent, libtree/src/lib/lib_tree.f90:405-431)
__global__ void k_tree_links(int nbox, int n, int nlev, const int* incl, const int* level_base, const int* run_start,
                             int* run_end, int* parent) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nbox) return;
    const int li = level_of_box(b, nlev, level_base);
    run_end[b] = (b + 1 < level_base[li + 1]) ? run_start[b + 1] : n;
    parent[b] = li > 0 ? incl[(int64_t)(li - 1) * n + run_start[b]] - 1 : -1;
}

__device__ __forceinline__ void deinterleave(long long nb, int l, long long c[3]) {
    c[0] = c[1] = c[2] = 0;
    for (int b = 0; b < l; ++b)
        for (int d = 0; d < 3; ++d) c[d] |= ((nb >> (3 * b + (2 - d))) & 1ll) << b;
}
__device__ __forceinline__ long long interleave(const long long c[3], int l) {
    long long nb = 0;
    for (int b = 0; b < l; ++b)
        for (int d = 0; d < 3; ++d) nb |= ((c[d] >> b) & 1ll) << (3 * b + (2 - d));
    return nb;
}
// the box and its neighbours at distance 1 inside [0, 2^l)^3, ascending
// (lib_tree_hf_get_neighbour_all_xD with k = 1, libtree/src/lib/lib_tree_helper_functions.f90:914-997)
__device__ inline int i2_sorted(long long nb, int l, long long* out) {
    long long c[3], q[3];
    deinterleave(nb, l, c);
    const long long hi = (1ll << l) - 1;
    int cnt = 0;
    for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dz = -1; dz <= 1; ++dz) {
                q[0] = c[0] + dx;
                q[1] = c[1] + dy;
                q[2] = c[2] + dz;
                if (q[0] < 0 || q[1] < 0 || q[2] < 0 || q[0] > hi || q[1] > hi || q[2] > hi) continue;
                out[cnt++] = interleave(q, l);
            }
    for (int a = 1; a < cnt; ++a) {   // insertion sort of at most 27 codes
        const long long v = out[a];
        int j = a - 1;
        while (j >= 0 && out[j] > v) {
            out[j + 1] = out[j];
            --j;
        }
        out[j + 1] = v;
    }
    return cnt;
}
// global id of box code nb among the level's boxes box_n[lo..hi) (ascending), or -1
__device__ __forceinline__ int find_box(const long long* box_n, int lo, int hi, long long nb) {
    const int end = hi;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (box_n[mid] < nb) lo = mid + 1;
        else hi = mid;
    }
    return (lo < end && box_n[lo] == nb) ? lo : -1;
}

// I4 = children of the parent's I2 minus the box's own I2, kept where the box exists, ascending
// (lib_tree_get_domain_i4, libtree/src/lib/lib_tree.f90:994-1143).  out == nullptr counts.
__global__ void k_tree_i4(int nbox, int nlev, const int* level_base, const long long* box_n, const int* box_level,
                          const int* ptr, int* cnt_out, int* out) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nbox) return;
    const int l = box_level[b];
    const int li = level_of_box(b, nlev, level_base);
    int cnt = 0;
    if (l > 0) {
        long long own[27], par[27];
        const int no = i2_sorted(box_n[b], l, own);
        const int np = i2_sorted(box_n[b] >> 3, l - 1, par);
        const int lo = level_base[li], hi = level_base[li + 1];
        int k = 0;   // own is ascending: walk it beside the ascending candidates
        for (int a = 0; a < np; ++a)
            for (int c = 0; c < 8; ++c) {
                const long long q = (par[a] << 3) | c;
                while (k < no && own[k] < q) ++k;
                if (k < no && own[k] == q) continue;
                const int id = find_box(box_n, lo, hi, q);
                if (id < 0) continue;
                if (out) out[ptr[b] + cnt] = id;
                ++cnt;
            }
    }
    if (!out) cnt_out[b] = cnt;
}

// E2 of leaf q = the runs of its own box and its existing neighbours, ascending box order
// (lib_tree_get_domain_e2, lib_tree.f90:611-724), sphere indices in input order.  out == nullptr counts.
__global__ void k_tree_e2(int nleaf, int leaf0, int nbox, int lmax, const long long* box_n, const int* run_start,
                          const int* run_end, const int* order, const int* ptr, int* cnt_out, int* out) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nleaf) return;
    const int b = leaf0 + q;
    long long own[27];
    const int no = i2_sorted(box_n[b], lmax, own);
    int cnt = 0;
    for (int a = 0; a < no; ++a) {
        const int id = find_box(box_n, leaf0, nbox, own[a]);
        if (id < 0) continue;
        for (int i = run_start[id]; i < run_end[id]; ++i) {
            if (out) out[ptr[q] + cnt] = order[i];
            ++cnt;
        }
    }
    if (!out) cnt_out[q] = cnt;
}

// Pass lists of the ML-FMM operator from the hierarchy, written into one buffer at the offsets
// lofs[0..11] of: aggregation (leaf <- its coupled spheres), children, I4, parent, box-to-sphere
// (sphere <- its leaf), near field (sphere <- E2 of its leaf without itself).  cnt_* are the
// per-item counts whose exclusive scans are the CSR pointers (written here with their totals).


__global__ void k_fmm_lists(FmmListArgs a) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int* L = a.list;
    // aggregation CSR over leaves
    if (t <= a.nleaf) L[a.lofs[0] + t] = a.agg_ptr[t];
    if (t < a.nleaf) {
        const int b = a.leaf0 + (int)t;
        int o = a.lofs[1] + a.agg_ptr[t];
        for (int i = a.run_start[b]; i < a.run_end[b]; ++i)
            if (a.couple[a.order[i]]) L[o++] = a.order[i];
    }
    // children: the boxes below level l_min in id order (their pointers: k_fmm_child_ptr)
    if (t == a.nbox) L[a.lofs[2] + t] = a.nbox - a.lb1;
    if (t < a.nbox - a.lb1) L[a.lofs[3] + t] = a.lb1 + (int)t;
    // I4 pointers (the ids are written by k_tree_i4)
    if (t <= a.nbox) L[a.lofs[4] + t] = a.i4_ptr[t];
    // parent CSR: boxes from l_min + 1 on have one parent each
    if (t <= a.nbox) L[a.lofs[6] + t] = t < a.lb1 ? 0 : (int)t - a.lb1;
    if (t < a.nbox - a.lb1) L[a.lofs[7] + t] = a.parent[a.lb1 + t];
    // box to sphere: sphere j <- its leaf
    if (t <= a.n) L[a.lofs[8] + t] = (int)t;
    if (t < a.n) L[a.lofs[9] + a.order[t]] = a.incl_leaf[t] - 1;
    // near field: sphere order[t] <- E2 of its leaf without itself
    if (t <= a.n) L[a.lofs[10] + t] = a.near_ptr[t];
    if (t < a.n) {
        const int j = a.order[t];
        const int q = a.incl_leaf[t] - 1 - a.leaf0;
        int o = a.lofs[11] + a.near_ptr[j];
        for (int e = a.e2_ptr[q]; e < a.e2_ptr[q + 1]; ++e)
            if (a.e2_idx[e] != j) L[o++] = a.e2_idx[e];
    }
}

// child pointers: box p's children are the boxes of the next level whose parent is p, a run in id
// order; ptr[p] = (first child id or, for a box without children, the id its children would start
// at) - lb1
__global__ void k_fmm_child_ptr(int nbox, int lb1, const int* parent, int* out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;   // child candidates c = lb1 .. nbox-1
    if (c < lb1 || c >= nbox) return;
    const int p = parent[c];
    const int pprev = (c > lb1) ? parent[c - 1] : -1;
    // every box in (pprev, p] starts its children at c
    for (int q = pprev + 1; q <= p; ++q) out[q] = c - lb1;
    if (c == nbox - 1)
        for (int q = p + 1; q < nbox; ++q) out[q] = nbox - lb1;
}

// per-sphere counts: near field |E2(leaf)| - 1; per-leaf counts: coupled spheres of the leaf
__global__ void k_fmm_counts(int n, int nleaf, int leaf0, const int* order, const int* couple, const int* incl_leaf,
                             const int* run_start, const int* run_end, const int* e2_cnt, int* near_cnt, int* agg_cnt) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) near_cnt[order[t]] = e2_cnt[incl_leaf[t] - 1 - leaf0] - 1;
    if (t < nleaf) {
        const int b = leaf0 + t;
        int c = 0;
        for (int i = run_start[b]; i < run_end[b]; ++i) c += couple[order[i]] ? 1 : 0;
        agg_cnt[t] = c;
    }
}

// box centres in the scene's units (lib_tree_get_centre_of_box, lib_tree.f90:1292-1300, unscaled by
// lib_tree_get_unscaled_point with D = max_d (x_max,d - x_min,d)(1 + 2^-52)), orders and offsets
__global__ void k_fmm_boxes(int nbox, const long long* box_n, const int* box_level, const double* mm, FmmLevels lv,
                            double* bc, int* bp, int64_t* bo) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nbox) return;
    double D = 0.0;
    for (int d = 0; d < 3; ++d) D = fmax(D, __dmul_rn(__dsub_rn(mm[3 + d], mm[d]), 1.0 + 2.220446049250313e-16));
    long long c[3];
    const int l = box_level[b];
    deinterleave(box_n[b], l, c);
    const double h = ldexp(1.0, -l);
    for (int d = 0; d < 3; ++d) bc[3 * (size_t)b + d] = __dadd_rn(__dmul_rn(__dmul_rn(h, __dadd_rn((double)c[d], 0.5)), D), mm[d]);
    const int li = l - lv.lmin;
    const int L = lv.order[li];
    bp[b] = L;
    bo[b] = lv.off[li] + (int64_t)(b - lv.base[li]) * 2 * L * (L + 2);
}

}  // namespace foggy
