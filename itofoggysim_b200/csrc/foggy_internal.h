// Internal declarations shared by the host (C++) and device (CUDA) parts of libfoggy_b200.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/foggy_gpu.h"

#ifdef __CUDACC__
#include <cuda_runtime.h>
#endif

namespace foggy {

// ---- host: 3j symbols and axial translation tables (gaunt.cpp) --------------------------
struct AxialTables {
    int pmax = 0;
    // offset[(m*(pmax+1) + n)*(pmax+1) + nu] = start of the q-list of (m, n, nu) in ga/gb,
    // q = 0..min(n, nu); -1 where undefined (n or nu < max(m, 1)).
    std::vector<int32_t> offset;
    std::vector<double> ga, gb;
};
int wigner3j_family(int j1, int j2, int m1, int m2, std::vector<double>& f);
double wigner3j(int j1, int j2, int j3, int m1, int m2, int m3);
void build_axial_tables(int pmax, AxialTables& t);
void build_axial_tables_qmajor(const AxialTables& t, std::vector<int64_t>& koff, std::vector<double>& gab);
void build_scalar_gaunt_qmajor(int NM, std::vector<int64_t>& koff, std::vector<double>& gs);
void build_g_table(int pmax, std::vector<double>& g);
void build_delta_table(int pmax, std::vector<double>& out);
// Raises a kernel's dynamic shared-memory ceiling to at least `bytes` on the current device.  The
// ceiling is a process-wide attribute of the function: handles launching the same kernel from
// several threads only ever raise it, under one lock, so no launch finds it lowered by another.
void raise_smem_ceiling(const void* func, size_t bytes);
// device bytes a direct solve will hold; pair tables counted when pair_tables == 1 (their size in
// *table_bytes either way)
int64_t estimate_solve_bytes(const foggy_params& prm, int N, const int* param_index, int NP, const int* n_range,
                             int pair_tables, int64_t* table_bytes);
// device bytes foggy_solve_block adds for a block of nrhs right-hand sides (its Krylov block,
// iterates, residuals and small arrays)
int64_t estimate_block_bytes(const foggy_params& prm, int N, const int* param_index, int NP, const int* n_range,
                             int nrhs);

// ---- host: octree box arithmetic (fmm_tree.cpp) ----------------------------------------------
// Level bounds of the ML-FMM's boxes (built on the device): levels l_min..l_max, boxes with a
// global id level by level in ascending Morton code.
struct FmmTree {
    int lmin = 0, lmax = 0;
    std::vector<int> level_base;           // first id of level lmin + i; level_base[nlev] = boxes
};
void morton_deinterleave(int64_t n, int l, int64_t c[3]);
int64_t morton_interleave(const int64_t c[3], int l);
void box_centre(int64_t n, int l, double out[3]);
// the box and its existing-or-not neighbours inside the domain (own box first), and the
// interaction list of box n at level l (ascending, every candidate inside the domain)
void tree_i2(int64_t n, int l, std::vector<int64_t>& out);
void tree_i4(int64_t n, int l, std::vector<int64_t>& out);

// Maximum truncation order of a sphere (the reference caps single spheres at 45,
// lib_mie_ss_helper_functions.f90:32).
constexpr int kMaxDegree = 45;

}  // namespace foggy

// ---- device-side views -------------------------------------------------------------------
#ifdef __CUDACC__
namespace foggy {

struct cplx {
    double x, y;
};
__host__ __device__ __forceinline__ cplx mk(double a, double b) { return cplx{a, b}; }
__host__ __device__ __forceinline__ cplx operator+(cplx a, cplx b) { return mk(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ cplx operator-(cplx a, cplx b) { return mk(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ cplx operator*(cplx a, cplx b) {
    return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ cplx operator*(double s, cplx a) { return mk(s * a.x, s * a.y); }
__host__ __device__ __forceinline__ cplx conjg(cplx a) { return mk(a.x, -a.y); }
// single-precision complex of the FP32 operator (the translation arithmetic of the mixed-precision
// solve); scalars of either precision multiply it in single precision
struct cplxf {
    float x, y;
};
__host__ __device__ __forceinline__ cplxf operator+(cplxf a, cplxf b) { return cplxf{a.x + b.x, a.y + b.y}; }
__host__ __device__ __forceinline__ cplxf operator-(cplxf a, cplxf b) { return cplxf{a.x - b.x, a.y - b.y}; }
__host__ __device__ __forceinline__ cplxf operator*(cplxf a, cplxf b) {
    return cplxf{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
__host__ __device__ __forceinline__ cplxf operator*(float s, cplxf a) { return cplxf{s * a.x, s * a.y}; }
__host__ __device__ __forceinline__ cplxf operator*(double s, cplxf a) { return (float)s * a; }
__host__ __device__ __forceinline__ cplxf conjg(cplxf a) { return cplxf{a.x, -a.y}; }
// complex of type C from two reals
template <class C>
__host__ __device__ __forceinline__ C cm(double a, double b) {
    return C{(decltype(C::x))a, (decltype(C::x))b};
}
__host__ __device__ __forceinline__ cplx cdiv(cplx a, cplx b) {
    // Smith's algorithm
    if (fabs(b.x) >= fabs(b.y)) {
        double r = b.y / b.x, d = b.x + b.y * r;
        return mk((a.x + a.y * r) / d, (a.y - a.x * r) / d);
    } else {
        double r = b.x / b.y, d = b.x * r + b.y;
        return mk((a.x * r + a.y) / d, (a.y * r - a.x) / d);
    }
}

// Sphere-major ragged layout of the device coefficient vectors: sphere j owns 2*P_j complex
// entries at off[j] (P_j = p_j (p_j + 2)): a-part (n = 1..p_j, m = -n..n) then b-part.
// Entries are scaled: device value = reference value / g_nm.
struct SceneView {
    int n;                     // spheres
    int pmax;                  // max p_j
    double k;                  // wavenumber
    const double* centres;     // 3n
    const int* p;              // n
    const int64_t* off;        // n + 1
    const cplx* an;            // n * pmax, a_n of sphere j at j*pmax + (n-1)
    const cplx* bn;
    const int* couple;         // n: 1 if the sphere's coupling rows are kept
};

struct AxialView {
    int pmax;
    const int32_t* offset;
    const double* ga;
    const double* gb;
    const int64_t* koff;   // q-major layout (build_axial_tables_qmajor)
    const double2* gab;
};

}  // namespace foggy
#endif
