// Kernel declarations of libfoggy_b200 (sm_100a).
#pragma once

#include <cuda_runtime.h>

#include "foggy_internal.h"

namespace foggy {

// Plane wave on the device (lib_mie_illumination.f90:392-478): propagation direction after
// the reference's cartesian round trip, Jones weights and phases, origin.
struct WaveDev {
    double kc[3];        // wave vector (cartesian)
    double alpha, beta;  // its polar and azimuthal angle
    double ax, phx;      // |J_x|, arg(J_x) + phase   (TM)
    double ay, phy;      // |J_y|, arg(J_y) + phase   (TE)
    double g;            // amplitude weight
    double d0[3];        // origin of the wave's coordinate system
};

// Hermite-Gaussian beam (lib_field_gaussian_beam_hermite_type, lib_field_gaussian_beam.f90:40-56,
// inside lib_mie_illumination_gaussian_beam_parameter, lib_mie_illumination.f90:58-93); its
// wavelength and medium are the solver's, e_field_0 = 1
struct GaussDev {
    double wx0, wy0;             // waist radii along x and y
    int tem_m, tem_n;            // Hermite-Gaussian mode
    double jxr, jxi, jyr, jyi;   // Jones vector
    double theta, phi;           // propagation direction of the beam axis
    double phase;                // extra phase
    double g;                    // amplitude weight
    double d0[3];                // origin of the beam coordinate system
    int convention;              // 1: exp(-i(kz - wt)), 2: exp(i(kz - wt))
};

// k_scene.cu
__global__ void k_mie_ab(int n_param, const double* size_param, const double* m_re, const double* m_im,
                         const int* p_of_param, int pstride, cplx* an_out, cplx* bn_out);
__global__ void k_gather_an(int n, const int* pidx, int pstride, const cplx* an_p, const cplx* bn_p,
                            cplx* an_s, cplx* bn_s);
__global__ void k_pitau(int nw, const WaveDev* waves, int pmax, double* pi_out, double* tau_out);
__global__ void k_rhs(SceneView sc, int nw, const WaveDev* waves, int pmax, const double* pi_tab,
                      const double* tau_tab, int nl, const WaveDev* lwaves, const double* lpi_tab,
                      const double* ltau_tab, cplx* b, cplx* pq);
__global__ void k_gauss_local(SceneView sc, int nb, const GaussDev* beams, double lambda0, double n_medium,
                              WaveDev* out);
__global__ void k_unpack(SceneView sc, int pg, const double* g, const cplx* xref, cplx* xdev);
__global__ void k_pack(SceneView sc, int pg, const double* g, const cplx* ydev, const cplx* identity_ref,
                       cplx* yref);
__global__ void k_cross_sections(SceneView sc, const cplx* x, const cplx* pq, double* part);
// scattered E, H at points (reference layout coefficients x, C entries per part and sphere)
__global__ void k_field(SceneView sc, const double* radius_s, int pg, int C, const cplx* x, const double* pts,
                        double e0, double h_factor, cplx* E_out, cplx* H_out);

// k_direct.cu -- all-pairs sphere coupling (the direct operator)
// Tables of the Wigner small-d recurrence (degrees <= K).
struct DTabs {
    const double* sqrt_binom;  // [J][m + K]: sqrt((2J)!/((J+m)!(J-m)!))
    const double* rs;          // [j][m]: sqrt(j^2 - m^2)
    const double* irs;         // [j][m]: 1/sqrt(j^2 - m^2) (0 for m = j)
    const double* rj;          // [2j] = 1/(j(j-1)), [2j+1] = 1/((j-1)(2j-1))
    int K;
};
// Scalar coaxial coefficients S(k; a, b) of every unordered sphere pair (s < t), computed once
// per scene and kept in HBM: block of pair u(s, t) = s N - s(s+1)/2 + t - s - 1 at pair_off[u],
// for k = 0..min(p_s, p_t) a square (M + 2 - k)^2 grid, M = max(p_s, p_t), over a, b = k..M+1,
// row-major (S is symmetric in a and b).
struct PairTabs {
    const cplx* stab;          // nullptr: the operator sums S from the Gaunt table per matvec
    const cplxf* stab32;       // the same in single precision (FP32 operator)
    const int64_t* pair_off;
};
struct SGaunt {
    const int64_t* koff;       // build_scalar_gaunt_qmajor layout
    const double* gs;
    int NM;
};
__host__ __device__ __forceinline__ int64_t pair_index(int s, int t, int n) {
    return (int64_t)s * n - (int64_t)s * (s + 1) / 2 + (t - s - 1);
}
// sum_{k' < k} (A - k')(B - k')
__host__ __device__ __forceinline__ int64_t pair_block_offset(int k, int A, int B) {
    int64_t kk = k;
    return kk * A * B - (int64_t)(A + B) * kk * (kk - 1) / 2 + (kk - 1) * kk * (2 * kk - 1) / 6;
}
__host__ __device__ __forceinline__ int64_t pair_block_size(int ps, int pt) {
    int km = ps < pt ? ps : pt;
    int M2 = (ps > pt ? ps : pt) + 2;
    return pair_block_offset(km + 1, M2, M2);
}
__global__ void k_pair_sizes(SceneView sc, int64_t* sizes);

struct DirectArgs {
    SceneView sc;
    DTabs dt;                  // rs[j][k] = sqrt(j^2 - k^2) for the coaxial relation
    const double* delta;       // d^j(pi/2), gaunt.cpp::build_delta_table layout
    const float* delta32;      // the same in single precision
    int fp32;                  // 1: the FP32 operator (stab32, delta32), FP64 input and slabs
    SGaunt g;                  // scalar Gaunt sums (no pair tables)
    PairTabs pt;
    int z;                     // radial function selector (1 j_n, 2 y_n, 3 h1, 4 h2)
    const cplx* x;             // ragged scaled input
    cplx* partial;             // [slabs][n_unk] partial sums
    int cmax;                  // slabs per source bucket
    int64_t n_unk;
};
// One launch: targets of one degree bucket against the sources of one degree bucket.
struct DirectBucket {
    const int* targets;
    int ntargets;
    const int* sources;
    int nsources;
    int slab;                  // first partial slab of this launch (slab + blockIdx.y)
    int chunks;                // CTAs per target (<= cmax)
    int pp;                    // largest degree of the launch (sizes shared memory)
};
size_t direct_smem_bytes(int pp, bool tabs, bool fp32 = false);
// Several right-hand sides: nrhs vectors of n_unk entries at x + r ld (ragged scaled layout); each
// launch adds T times its (target bucket <- source bucket) sum onto y + r ld.  d carries the scene
// and tables (d.fp32 selects the FP32 operator); d.x, d.partial and d.cmax are not used.
struct BlockArgs {
    DirectArgs d;
    const cplx* x;
    cplx* y;
    int nrhs;
    int64_t ld;
};
// shared memory of one CTA of the several-right-hand-side operator with R vectors per CTA
size_t block_smem_bytes(int pp, bool tabs, bool fp32, int R);
// false when R is not one of the built tile widths (FP32: 1, 2, 4, 8, 16; FP64: 1, 2, 4, 8)
bool launch_direct_block(const BlockArgs& a, const DirectBucket& b, int R, cudaStream_t s);
size_t translation_pair_smem_bytes(int pmax);
void launch_direct(const DirectArgs& a, const DirectBucket& b, cudaStream_t s);

// k_pair_tables.cu -- the pair tables over groups of pairs with one M2 = max order + 2: FP32 as
// tensor-core products (tcgen05 kind::tf32, 3xTF32; the group's pairs share the Gaunt operand, a
// tile is up to np pairs), FP64 summed on the CUDA cores (tiles of up to kPairs64 pairs).
struct TcGroup {
    int M2, K, np;        // K: degrees p = 0..2 M2 - 2 padded to 8; np: pairs per tile (64, or 16 for K > 72)
    int mtiles;           // 128-row tiles of the packed Gaunt operand (the group's largest block)
    int64_t a_off;        // float offset of the group's packed operand
};
struct TcTile {
    int group, first, count;   // pairs first..first + count - 1 of the sorted pair list
    int m0, m1;                // the 128-row tiles m0..m1 - 1 of their blocks (at most 8)
};
struct TcArgs {
    SceneView sc;
    int z;
    const int2* pairs;         // (s, t), s < t, by group, largest block first within a group
    const TcTile* tiles;
    const TcGroup* groups;
    const float* a;            // packed Gaunt operands
    const int64_t* pair_off;
    cplxf* stab;
    int* err;                  // set when a wait for a copy or the tensor core timed out
};
int64_t tc_group_rows(int M2);
int tc_group_k(int M2);
int tc_group_pairs(int K);
size_t tc_smem_bytes(int K, int np);
void launch_tc_pack_a(SGaunt g, const TcGroup& gr, float* out, cudaStream_t s);
void launch_pair_tc(const TcArgs& a, int tile0, int ntiles, int K, int np, cudaStream_t s);
constexpr int kPairs64 = 32;   // pairs per tile of the FP64 tables
struct PairArgs {
    SceneView sc;
    int z;
    const int2* pairs;
    const TcTile* tiles;       // tiles of up to kPairs64 pairs, runs of up to 16 row tiles
    const TcGroup* groups;
    SGaunt g;
    const int64_t* pair_off;
    cplx* stab;
};
size_t pair_s_group_smem_bytes(int M2);
void launch_pair_s_group(const PairArgs& a, int tile0, int ntiles, int M2, cudaStream_t s);
// y = x + T (sum of the slab partials) for coupled spheres, y = x otherwise
__global__ void k_direct_finish(SceneView sc, const cplx* x, const cplx* partial, int slabs, int64_t n_unk,
                                cplx* y);
// Sphere or box centres with their truncation orders and the offsets of their coefficient
// vectors (scaled basis, a then b, standard (n, m) order).
struct PointSet {
    const double* c;
    const int* p;
    const int64_t* off;
};
// One ML-FMM pass: targets tbase .. tbase + n - 1 of tgt, target tbase + b translating its sources
// lidx[lptr[b] .. lptr[b+1]) of src by t = k (sign (c_src - c_tgt) + sh) with radial function z;
// the result is written to (add = 0) or added onto (add = 1) out + tgt.off[target].
struct TransArgs {
    PointSet tgt, src;
    const cplx* x;
    cplx* out;
    const int* lptr;
    const int* lidx;
    int tbase;
    double k, sign, sh[3];
    int z, add, pp;
    const double* delta;
    DTabs dt;
    SGaunt g;
    cplx* slab;        // chunks > 1: partial sums, chunk c of target i at slab + (c ntargets + i) slab_ld
    int64_t slab_ld;   // >= 2 P of every target of the pass
    const cplx* tab;         // coaxial blocks of the pass's translations (k_fmm_tab), or null:
    const int64_t* tab_off;  // entry i's block at tab + tab_off[i] (aligned with lidx)
    int fp32;                // translation arithmetic in single precision (mixed-precision Arnoldi
    const float* delta32;    // steps): d^j(pi/2) and the blocks in FP32, coefficients kept in FP64
    const cplxf* tab32;
};
__global__ void k_narrow(const cplx* in, cplxf* out, int64_t n);
// a distinct translation of an ML-FMM pass: its length, degrees and block offset in the tables
struct FmmTabEntry {
    double rho;
    int pt, ps;
    int64_t off;
};
__global__ void k_fmm_rho(TransArgs a, double* rho, int2* deg);
__global__ void k_fmm_tab(const FmmTabEntry* u, SGaunt g, int z, cplx* tab);
// one pass: ntargets x chunks CTAs (chunks >= 1; with several, slab must hold chunks x ntargets x
// slab_ld entries)
void launch_translate(const TransArgs& a, int ntargets, int chunks, cudaStream_t s);
// single-pair translation for the parity entry point: A, B blocks in the scaled basis
__global__ void k_translation_pair(AxialView ax, DTabs dt, double x, double theta, double phi, int pn, int pnu,
                                   int z, cplx* A, cplx* B);

// k_gmres.cu -- Krylov kernels (deterministic fixed-order reductions)
constexpr int kRedBlocks = 296;
__global__ void k_dots_partial(const cplx* V, int64_t ld, int nv, const cplx* w, int64_t n, cplx* part);
__global__ void k_dots_reduce(const cplx* part, int nv, cplx* out, int accumulate);
__global__ void k_axpy_multi(const cplx* V, int64_t ld, int nv, const cplx* h, cplx* w, int64_t n);
__global__ void k_norm_partial(const cplx* w, int64_t n, double* part);
__global__ void k_norm_reduce(const double* part, double* out);
__global__ void k_scale_copy(const cplx* w, const double* nrm, cplx* v, int64_t n);
__global__ void k_sub(const cplx* b, const cplx* ax, cplx* r, int64_t n);
__global__ void k_givens(cplx* H, int ldh, cplx* cs, double* sn, cplx* g, const cplx* h, const cplx* c,
                         const double* hn, int k, double* res_est, int* flags);
__global__ void k_trisolve(const cplx* H, int ldh, const cplx* g, int k, cplx* y);
__global__ void k_update_x(cplx* x, const cplx* V, int64_t ld, const cplx* y, int k, int64_t n);
__global__ void k_init_cycle(cplx* g, int m1, const double* beta, int* flags);
// several right-hand sides: one Krylov space per slot (blockIdx.y), basis vector i of slot b at
// V + i ldi + b ld; live[b] = 0 skips a slot that has left the restart cycle
__global__ void k_dots_partial_b(const cplx* V, int64_t ldi, int64_t ld, int nv, const cplx* W, int64_t n,
                                 const int* live, cplx* part);
__global__ void k_dots_reduce_b(const cplx* part, int nv, const int* live, cplx* out, int ostride);
__global__ void k_axpy_multi_b(const cplx* V, int64_t ldi, int64_t ld, int nv, const cplx* h, int hstride, cplx* W,
                               int64_t n, const int* live);
__global__ void k_norm_partial_b(const cplx* W, int64_t ld, int64_t n, const int* live, double* part);
__global__ void k_norm_reduce_b(const double* part, const int* live, double* out, int ostride);
__global__ void k_scale_copy_b(const cplx* W, int64_t ldw, const double* nrm, int nstride, cplx* Vout, int64_t ldv,
                               int64_t n, const int* live);
__global__ void k_sub_b(const cplx* Bv, const cplx* AX, cplx* Rv, int64_t ld, int64_t n);
__global__ void k_init_cycle_b(cplx* g, int m1, const double* beta, int nslots, int* live, int* kend);
__global__ void k_givens_b(cplx* H, int m, cplx* cs, double* sn, cplx* g, const cplx* h, const cplx* c,
                           const double* hn, int k, const double* tol_abs, double* res_est, int* flags, int* live,
                           int* kend, int nslots);
__global__ void k_trisolve_b(const cplx* H, int m, const cplx* g, const int* kend, cplx* y, int nslots);
__global__ void k_update_x_b(cplx* X, int64_t ld, const cplx* V, int64_t ldi, const cplx* y, int ystride,
                             const int* kend, int64_t n);

// k_tree.cu -- octree keys (libtree)
__global__ void k_minmax(int n, const double* c, double* out);
__global__ void k_morton(int n, const double* c, const double* mm, unsigned long long* key, int* idx);
__global__ void k_level_max(int n, int s, const unsigned long long* key, int* lmax);
__global__ void k_uindex_points(int n, const double* pts, int l, long long* out);
// ML-FMM hierarchy and pass lists from the sorted keys (all on the device)
__global__ void k_tree_flags(int n, int nlev, int lmin, const unsigned long long* key, int* flag);
__global__ void k_tree_boxes(int n, int nlev, int lmin, const unsigned long long* key, const int* incl,
                             long long* box_n, int* box_level, int* run_start, int* level_base);
__global__ void k_tree_links(int nbox, int n, int nlev, const int* incl, const int* level_base, const int* run_start,
                             int* run_end, int* parent);
__global__ void k_tree_i4(int nbox, int nlev, const int* level_base, const long long* box_n, const int* box_level,
                          const int* ptr, int* cnt_out, int* out);
__global__ void k_tree_e2(int nleaf, int leaf0, int nbox, int lmax, const long long* box_n, const int* run_start,
                          const int* run_end, const int* order, const int* ptr, int* cnt_out, int* out);
struct FmmListArgs {
    int n, nbox, nleaf, leaf0, lb1;
    const int* order;
    const int* couple;
    const int* incl_leaf;
    const int* run_start;
    const int* run_end;
    const int* parent;
    const int* e2_ptr;
    const int* e2_idx;
    const int* agg_ptr;
    const int* i4_ptr;
    const int* near_ptr;
    int lofs[12];
    int* list;
};
__global__ void k_fmm_lists(FmmListArgs a);
__global__ void k_fmm_child_ptr(int nbox, int lb1, const int* parent, int* out);
__global__ void k_fmm_counts(int n, int nleaf, int leaf0, const int* order, const int* couple, const int* incl_leaf,
                             const int* run_start, const int* run_end, const int* e2_cnt, int* near_cnt, int* agg_cnt);
// expansion order, coefficient offset and first box id per level (index l - lmin)
struct FmmLevels {
    int lmin;
    int order[22];
    int base[22];
    int64_t off[22];
};
__global__ void k_fmm_boxes(int nbox, const long long* box_n, const int* box_level, const double* mm, FmmLevels lv,
                            double* bc, int* bp, int64_t* bo);

}  // namespace foggy
