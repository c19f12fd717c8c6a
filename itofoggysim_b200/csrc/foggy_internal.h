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
