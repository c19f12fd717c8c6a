/*
 * foggy_gpu.h -- C ABI of the B200 multi-sphere Mie solver (sm_100a, one GPU).
 *
 * This is the drop-in boundary for ItoFoggySim's multi-sphere solve.  Each entry point
 * replaces one reference interface; the citation beside it is the reference file:line
 * (paths relative to the reference project root).  A Fortran caller binds these through
 * iso_c_binding (itofoggysim_b200/fortran/foggy_gpu_f.f90), Python through ctypes
 * (itofoggysim_b200/_native.py).
 *
 * Conventions
 *   - every call returns FOGGY_OK (0) or a negative status; foggy_last_error() explains it;
 *   - complex numbers are two interleaved doubles (Fortran complex(8), C double _Complex);
 *   - coefficient vectors use the reference's flat layout: per sphere i (in input order)
 *     a block of 2*C complex entries, C = (n2+1)^2 - n1^2 for the global n_range [n1,n2]:
 *     first a_nm for n = n1..n2, m = -n..n, then b_nm in the same order
 *     (FoggySim/src/lib/mie_theory/lib_mie_ms_solver_interface_helper_functions.f90:49-163);
 *     entries above a sphere's own truncation order are zero;
 *   - pointers flagged FOGGY_MEM_HOST are ordinary host memory, FOGGY_MEM_DEVICE are CUDA
 *     device pointers on the handle's device; all buffers are caller-owned;
 *   - lengths are in one unit of the caller's choice (the reference uses metres); the
 *     wavenumber is k = 2*pi*n_medium/lambda_0.
 *   - a handle is used by one host thread at a time; it owns one CUDA stream.
 */
#ifndef FOGGY_GPU_H
#define FOGGY_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ----------------------------------------------------------------- */
#define FOGGY_OK                 0
#define FOGGY_ERR_ARGUMENT      -1   /* invalid argument or size                        */
#define FOGGY_ERR_STATE         -2   /* call out of order (e.g. solve before spheres)   */
#define FOGGY_ERR_CUDA          -3   /* a CUDA runtime call failed                      */
#define FOGGY_ERR_NOMEM         -4   /* the solve does not fit the device memory budget */
#define FOGGY_ERR_NOT_CONVERGED -5   /* GMRES stopped at max_iterations above tolerance */
#define FOGGY_ERR_BREAKDOWN     -6   /* GMRES breakdown (zero Krylov vector)            */
#define FOGGY_ERR_NAN           -7   /* NaN or Inf met in the residual                  */
#define FOGGY_ERR_UNSUPPORTED   -8   /* option not built                                */

#define FOGGY_MEM_HOST   0
#define FOGGY_MEM_DEVICE 1

#define FOGGY_MATVEC_DIRECT 0   /* all sphere pairs (..._without_transposed_all)        */
#define FOGGY_MATVEC_MLFMM  1   /* multilevel FMM (lib_mie_ms_ml_fmm_calculate_vector_b) */

typedef struct foggy_handle_s* foggy_handle;

/* Solver configuration.  Mirrors the Fortran state the reference keeps in
 * simulation_data%spherical_harmonics (FoggySim/src/lib/mie_theory/lib_mie_type.f90:43-99),
 * lib_mie_ms_solver_parameter_type (lib_mie_ms_solver_interface.f90:63-67) and
 * solver_gmres_parameter_type (lib_solver_GMRES.f90:39-50). */
typedef struct foggy_params {
    double  lambda_0;            /* vacuum wavelength                                       */
    double  n_medium;            /* refractive index of the medium (real)                   */
    int32_t n_range[2];          /* global degree range [n1, n2], n1 >= 1                   */
    int32_t z_coupling;          /* radial function of the sphere-sphere translation:
                                    1 = j_n (the reference's z_selector_incident_wave in all of
                                    its tests), 3 = h_n^(1) (scattered-wave coupling)       */
    int32_t reference_row_rule;  /* 1: zero the coupling rows of a sphere whose n_range does
                                    not cover the global n_range, as the reference does
                                    (lib_mie_ms_solver_interface.f90:965-978); 0: couple every
                                    sphere up to its own truncation order                  */
    int32_t matvec_mode;         /* FOGGY_MATVEC_DIRECT or FOGGY_MATVEC_MLFMM                */
    int32_t use_initial_guess;   /* 1: x0 = single-sphere solution a_n p, b_n q            */
    int32_t gmres_restart;       /* Krylov dimension per restart cycle (reference: 10)      */
    int32_t gmres_max_iterations;/* reference: 1000                                        */
    double  gmres_tolerance;     /* stop when ||b - A x|| / ||b|| <= tolerance              */
    int32_t tree_l_max;          /* 0: reference rule from tree_s_opt; > 0: fixed deepest level */
    int32_t tree_s_opt;          /* elements per leaf for the reference l_max rule (10)     */
    double  fmm_digits;          /* ML-FMM box orders: 0 = the global order n_range(2) on every
                                    level, as the reference does; d > 0 = per level the
                                    excess-bandwidth order kd + 1.8 d^(2/3) (kd)^(1/3) of the
                                    box diagonal d, rounded up, never below the global order,
                                    at most 45 (not in the reference)                      */
    int64_t device_memory_budget;/* bytes the handle may allocate; 0 = 90% of free memory  */
    int32_t pair_tables;         /* geometry-only scalar translation coefficients of every sphere
                                    pair kept in device memory for the solve: 0 = when they fit
                                    beside the Krylov basis, 1 = always, -1 = never (the
                                    operator sums them on every application)               */
    int32_t fmm_convention;      /* ML-FMM translations: 0 = as the reference writes them
                                    (lib_mie_ms_ml_fmm_interface.f90:259-981: z_coupling for
                                    every box translation, box-to-sphere with
                                    z_translation_gt_r, its displacement signs, and the
                                    box-to-sphere offset of lib_tree_get_unscaled_point);
                                    1 = consistent expansion (regular translations up and down
                                    the tree, z_coupling across the interaction lists), which
                                    tends to the direct operator as the order grows        */
    int32_t z_translation_gt_r;  /* radial function of the box-to-sphere step in convention 0
                                    (the reference's tests set 3)                          */
    int32_t precision;           /* 0: FP64 throughout; 1: mixed: the Arnoldi steps apply the
                                    operator (direct or ML-FMM) in FP32 (single-precision
                                    coaxial blocks, rotations and coaxial sums; FP64 vectors
                                    and box coefficients), the true residual at the start and
                                    at every restart in FP64, so the restarts refine to
                                    gmres_tolerance.  foggy_matvec stays FP64.               */
} foggy_params;

/* Per-solve statistics (the reference prints these; here they are returned). */
typedef struct foggy_stats {
    int32_t iterations;          /* Arnoldi steps performed                                 */
    int32_t restarts;
    int32_t matvecs;
    int32_t status;              /* FOGGY_OK or FOGGY_ERR_NOT_CONVERGED / _BREAKDOWN / _NAN */
    double  backward_error;      /* final true ||b - A x|| / ||b||                         */
    double  ms_total;            /* device time of the solve                                */
    double  ms_matvec;           /* device time inside the matvec                           */
    double  ms_setup;            /* translation tables, Mie coefficients, right-hand side    */
    int64_t kernel_launches;     /* CUDA kernels this library launched during the solve     */
} foggy_stats;

/* ---- lifecycle ------------------------------------------------------------------------ */

/* Fills *p with the reference defaults (lib_mie_ms_constructor, lib_mie_multi_sphere.f90:111-150;
 * lib_mie_ms_solver_gmres_get_parameter_std_values, lib_solver_GMRES.f90:93-106). */
void foggy_default_params(foggy_params* p);

/* Replaces lib_mie_ms_constructor + lib_mie_ms_solver_constructor
 * (lib_mie_multi_sphere.f90:111-150, lib_mie_ms_solver_interface.f90:91-129). */
int32_t foggy_create(const foggy_params* params, int32_t device, foggy_handle* out);

/* Replaces lib_mie_ms_solver_destructor (lib_mie_ms_solver_interface.f90:131-141). */
int32_t foggy_destroy(foggy_handle h);

/* Message of the last failing call on this handle; with h = NULL, of the calling thread's last
 * failing foggy_create or handle-less call. */
const char* foggy_last_error(foggy_handle h);

/* Replaces lib_mie_ms_solver_set_n_range / _set_max_iterations / _use_ml_fmm
 * (lib_mie_ms_solver_interface.f90:156-201). */
int32_t foggy_set_params(foggy_handle h, const foggy_params* params);

/* ---- scene ---------------------------------------------------------------------------- */

/* Sphere list and shared sphere parameters; replaces filling simulation_data%sphere_list and
 * %sphere_parameter_list through lib_mie_type_func_get_sphere_parameter
 * (FoggySim/src/lib/mie_theory/lib_mie_type_functions.f90:46-86).
 *   centres[3*n_spheres]         d_0_j, x y z per sphere
 *   param_index[n_spheres]       0-based index into the parameter arrays
 *   refractive_index[2*n_param]  complex particle index (re, im)
 *   radius[n_param]
 *   n_range[2*n_param]           per-parameter degree range [1, n_max] (n_max <= global n2)
 * Mie coefficients a_n, b_n are computed on the device in FP64. */
int32_t foggy_set_spheres(foggy_handle h, int32_t n_spheres, const double* centres,
                          const int32_t* param_index, int32_t n_param,
                          const double* refractive_index, const double* radius,
                          const int32_t* n_range);

/* Plane-wave illumination; replaces lib_mie_type_func_get_plane_wave_illumination
 * (lib_mie_type_functions.f90:122-167) with the Jones vector and phase of
 * lib_mie_illumination_get_p_q_j_j_multi_plane_wave (lib_mie_illumination.f90:392-478).
 *   theta[nw], phi[nw]   propagation direction of wave i
 *   jones[4*nw]          (re x, im x, re y, im y): x -> TM part, y -> TE part
 *   g[nw]                amplitude weight, phase[nw] extra phase
 *   d_0_i[3*nw]          origin of the wave's coordinate system
 * All waves of one call form ONE right-hand side, as in the reference. */
int32_t foggy_set_plane_waves(foggy_handle h, int32_t nw, const double* theta, const double* phi,
                              const double* jones, const double* g, const double* phase,
                              const double* d_0_i);

/* Gaussian beams illuminating the cluster, added to the plane waves (lib_mie_illumination_get_p_q_j_j,
 * lib_mie_illumination.f90:206-250); nb = 0 removes them.  The reference's working beam model,
 * the plane-wave approximation (calculation_type 3, lib_mie_illumination_get_p_q_gaussian_beam,
 * lib_mie_illumination.f90:781-918, with lib_field_gaussian_beam_hermite_get_plane_wave_approximation,
 * FoggySim/src/lib/field/lib_field_gaussian_beam.f90:256-358): each sphere sees the plane wave
 * along the beam's local phase gradient, with its local phase and projected polarisation.  Per
 * beam: waist radii x0, y0 (waist[2 nb]), Hermite-Gaussian mode m, n (tem[2 nb], 0..30), axis
 * direction theta, phi, Jones vector (jones[4 nb]: re x, im x, re y, im y), weight g (applied
 * twice, as the reference does), phase (NULL = 0), origin d_0_i[3 nb] (NULL = 0) and time
 * convention (convention[nb], 1 or 2; NULL = 1).  The beams use the handle's lambda_0 and
 * n_medium.  Setting plane waves with nw = 0 leaves only the beams. */
int32_t foggy_set_gaussian_beams(foggy_handle h, int32_t nb, const double* waist, const int32_t* tem,
                                 const double* theta, const double* phi, const double* jones, const double* g,
                                 const double* phase, const double* d_0_i, const int32_t* convention);

/* Number of complex entries of one coefficient vector in the reference layout. */
int64_t foggy_vector_length(foggy_handle h);

/* ---- parity / building blocks ---------------------------------------------------------- */

/* Mie coefficients a_n, b_n for parameter set ip, n = n1..n2 of that parameter
 * (lib_mie_ss_helper_functions.f90:628-722).  a, b: complex[n2-n1+1], host memory. */
int32_t foggy_get_mie_coefficients(foggy_handle h, int32_t ip, double* a, double* b);

/* Right-hand side b = [a_n p_nm ; b_n q_nm] per sphere
 * (lib_mie_ms_solver_get_vector_b_all, lib_mie_ms_solver_interface.f90:230-315). */
int32_t foggy_get_vector_b(foggy_handle h, double* b, int32_t mem);

/* y = A x (lib_mie_ms_solver_calculate_vector_b, lib_mie_ms_solver_interface.f90:739-783,
 * direct form 806-998; ML-FMM form lib_mie_ms_ml_fmm_calculate_vector_b,
 * lib_mie_ms_ml_fmm_interface.f90:110-176). */
int32_t foggy_matvec(foggy_handle h, const double* x, double* y, int32_t mem);

/* Solve A x = b by restarted GMRES on the device; replaces lib_mie_ms_solver_run and
 * lib_mie_ms_solver_gmres_run (lib_mie_ms_solver_interface.f90:143-154,
 * lib_solver_GMRES.f90:116-316).  x0 may be NULL (then the params' use_initial_guess
 * decides between 0 and the single-sphere solution).  stats may be NULL. */
int32_t foggy_solve(foggy_handle h, const double* x0, double* x, int32_t mem, foggy_stats* stats);

/* Backward error of the last solve (lib_mie_ms_solver_get_backward_error, :203-209). */
double foggy_get_backward_error(foggy_handle h);

/* Extinction, scattering and absorption cross-sections of the whole cluster for the
 * coefficient vector x (reference layout).  The reference has only the single-sphere form
 * (lib_mie_ss_helper_functions.f90:1380-1475); the cluster form sums Xu's per-sphere
 * extinction and absorption terms. out[3] = {C_sca, C_ext, C_abs}. */
int32_t foggy_cross_sections(foggy_handle h, const double* x, int32_t mem, double* out);

/* Vector translation coefficients A_mn^{mu nu}, B_mn^{mu nu} at kd = x, direction (theta,
 * phi), computed on the device by rotation + axial translation + rotation back; replaces
 * lib_math_vector_spherical_harmonics_translation_coeff_r
 * (libmath/src/math/lib_math_vector_spherical_harmonics.f90:1354-1585).
 * A, B: host complex[C_n * C_nu], row (n, m) major, C_n = (n2+1)^2-n1^2. */
int32_t foggy_translation_coefficients(double x, double theta, double phi,
                                       const int32_t n_range[2], const int32_t nu_range[2],
                                       int32_t z_selector, double* A, double* B);

/* Wigner 3j symbol (j1 j2 j3; m1 m2 m3) for integer arguments; replaces lib_math_wigner_3j
 * (libmath/src/math/lib_math_wigner.f90:45-72, which calls wigxjpf).  Host computation by the
 * three-term recurrence that also builds the device's axial translation tables. */
double foggy_wigner_3j(int32_t j1, int32_t j2, int32_t j3, int32_t m1, int32_t m2, int32_t m3);

/* ---- octree (libtree) ------------------------------------------------------------------ */

/* Builds the octree of the sphere centres on the device; replaces lib_tree_constructor
 * (libtree/src/lib/lib_tree.f90:147-270).  Outputs (each may be NULL):
 *   uindex_out[n_spheres]  universal index of each sphere at level l_max (input order)
 *   order_out[n_spheres]   sphere indices sorted by their level-21 universal index
 *   l_min_out, l_max_out   level range (lib_tree_get_level_min/max, lib_tree.f90:1162-1242) */
int32_t foggy_build_tree(foggy_handle h, int64_t* uindex_out, int32_t* order_out,
                         int32_t* l_min_out, int32_t* l_max_out);

/* Universal index of points already scaled to [0,1)^3 at level l (1..21); replaces
 * lib_tree_hf_get_universal_index (libtree/src/lib/lib_tree_helper_functions.f90:202-364).
 * points[3*n] host memory, out[n]. */
int32_t foggy_universal_index(int32_t n, const double* points, int32_t l, int64_t* out);

/* Device bytes a direct-operator solve of this scene holds at its peak, from the plan the handle
 * follows (scene arrays, operator slabs, Krylov workspace, staging, order tables), into
 * solve_bytes, and the pair tables' bytes into table_bytes (FP64, plus FP32 when
 * params->precision = 1).  The solve server admits requests by these.  Host only: no handle, no
 * GPU. */
int32_t foggy_estimate_solve_bytes(const foggy_params* params, int32_t n_spheres, const int32_t* param_index,
                                   int32_t n_param, const int32_t* n_range, int64_t* solve_bytes,
                                   int64_t* table_bytes);

/* libtree box arithmetic on universal indices (box n at level l, 0 <= n < 8^l, l = 0..21), on the
 * host: no handle, no GPU.
 * foggy_tree_parent: the box `step` levels up (1 <= step <= l), n >> 3 step
 *   (lib_tree_get_parent, libtree/src/lib/lib_tree.f90:405-431).
 * foggy_tree_children: the eight boxes 8 n + j, j = 0..7, at level l + 1 (l < 21)
 *   (lib_tree_get_children, lib_tree.f90:444-453).
 * foggy_tree_centre_of_box: centre[3] = 2^-l (c + 1/2) in the normalised cube [0,1)^3, c the
 *   de-interleaved box coordinates (lib_tree_get_centre_of_box, lib_tree.f90:1292-1300).
 * foggy_tree_neighbours: the boxes at distance 1 inside the domain, ascending, out[26] at most
 *   (lib_tree_hf_get_neighbour_all_xD with k = 1, lib_tree_helper_functions.f90:914-997). */
int32_t foggy_tree_parent(int64_t n, int32_t l, int32_t step, int64_t* parent);
int32_t foggy_tree_children(int64_t n, int32_t l, int64_t* children);
int32_t foggy_tree_centre_of_box(int64_t n, int32_t l, double* centre);
int32_t foggy_tree_neighbours(int64_t n, int32_t l, int64_t* out, int32_t* count);

/* Number of boxes at tree level l and their universal indices in ascending order
 * (lib_ml_fmm_hf_create_hierarchy, libmlfmm/src/lib/lib_ml_fmm_helper_functions.f90:366-457).
 * Call with boxes == NULL to query the count. */
int32_t foggy_tree_boxes(foggy_handle h, int32_t l, int64_t* boxes, int32_t* count);

/* Scattered electric and magnetic field of the cluster at npoints points (3 doubles each):
 * replaces lib_mie_ms_get_field (FoggySim/src/lib/mie_theory/lib_mie_multi_sphere.f90:379-434)
 * with lib_mie_ss_get_field per sphere (lib_mie_single_sphere.f90:1397-1582) and the vector
 * spherical wave functions of lib_math_vector_spherical_harmonics_components_real_xu
 * (libmath/src/math/lib_math_vector_spherical_harmonics.f90:132-419): x holds the coefficients
 * a_nm, b_nm in the reference layout, e_field_0 the amplitude |E0|; e_out and h_out receive 3
 * complex cartesian components per point (H includes n_medium / c0).  Both fields are zero at a
 * point inside any sphere, as in the reference.  mem applies to x, points, e_out and h_out. */
int32_t foggy_get_field(foggy_handle h, const double* x, int32_t mem, int32_t npoints, const double* points,
                        double e_field_0, double* e_out, double* h_out);

/* Octree lists of box n at level l for the ML-FMM: kind 1 -> E1, the spheres in the box
 * (lib_tree_get_domain_e1, libtree/src/lib/lib_tree.f90:492-609); kind 2 -> E2, the spheres in
 * the box and its neighbours (lib_tree_get_domain_e2, :611-724); kind 4 -> I4, the level-l box
 * indices of the interaction list, every candidate inside the domain (lib_tree_get_domain_i4,
 * :994-1143).  Spheres are 0-based input indices in key order, boxes ascending.  Call with
 * out == NULL to query the count. */
int32_t foggy_tree_domain(foggy_handle h, int32_t l, int64_t n, int32_t kind, int64_t* out, int32_t* count);

/* The ML-FMM's pass lists as the library builds them on the device from the sorted keys (the
 * reference builds them in lib_ml_fmm_hf_create_hierarchy, libmlfmm/src/lib/lib_ml_fmm_helper_functions.f90:366-457,
 * with lib_tree_get_domain_e1/e2/i4, libtree/src/lib/lib_tree.f90:492-1143), one CSR list per part:
 * 0/1 aggregation (leaf box <- its coupled spheres), 2/3 children, 4/5 interaction list I4 (existing
 * boxes), 6/7 parent, 8/9 box to sphere (sphere <- its leaf box), 10/11 near field (sphere <- E2 of
 * its leaf without itself); even parts are pointers, odd parts indices.  Boxes are numbered level by
 * level from l_min in ascending universal index, leaf pointers run over the leaf boxes in that order,
 * spheres are 0-based input indices.  out = NULL queries the length. */
int32_t foggy_fmm_lists(foggy_handle h, int32_t part, int32_t* out, int32_t* count);

/* ---- operator without allocation ------------------------------------------------------- */

/* y = A x for device buffers x, y (reference layout), the direct operator only, with no
 * device-memory allocation.  This entry point has no counterpart in the reference.
 *
 * It serves callers that must not call cudaMalloc once their set-up is done: an outer
 * iteration (for example an eigen- or time-stepping loop, or another code's Krylov solver)
 * that runs under a memory pool owning the rest of the GPU, or that has been checked to make
 * no allocation after warm-up.  foggy_matvec may allocate staging buffers and, on its first
 * call, the pair coefficient tables; this one only uses what foggy_set_spheres made and a
 * fixed 32 MiB array of device memory that is part of the library, present on every GPU the
 * library is loaded on until the process exits.  Pair tables that an earlier foggy_matvec
 * or foggy_solve built on this handle are read, never built here.
 *
 * Limit: the scene's working memory, 16 * n * (2 + b) bytes for n scaled unknowns
 * (sum over spheres of 2 p (p + 2)) and b truncation-order buckets of 4 degrees, must fit
 * in 32 MiB; larger scenes return FOGGY_ERR_ARGUMENT and must use foggy_matvec.  Modes other
 * than FOGGY_MATVEC_DIRECT return FOGGY_ERR_UNSUPPORTED.
 *
 * The first call on a GPU looks up the array's device address (cudaGetSymbolAddress) with
 * that GPU current; make that first call before any stream capture.  All calls on one GPU
 * share the array, from every handle and thread: calls whose work overlaps on the GPU (other
 * streams, other threads) race and give wrong results.  The call returns after its work has
 * finished on the handle's stream. */
int32_t foggy_matvec_static(foggy_handle h, const double* x, double* y);

/* ---- several right-hand sides --------------------------------------------------------- */

/* One solve per plane wave set on the handle (nrhs must equal that count; no Gaussian beams):
 * right-hand side r is the incidence of wave r alone, as the reference obtains it by running
 * lib_mie_ms_solver_run once per illumination (lib_mie_ms_solver_interface.f90:143-154).  The
 * operator and its pair tables are built once and shared.  x (and x0, if not NULL) hold nrhs
 * vectors of foggy_vector_length entries one after the other; cross_sections (NULL to skip)
 * receives {C_sca, C_ext, C_abs} per right-hand side.  stats sums iterations, restarts,
 * matvecs and times over the solves, with the largest backward error; the status is that of the
 * first solve that did not converge, or FOGGY_OK. */
int32_t foggy_solve_rhs(foggy_handle h, int32_t nrhs, const double* x0, double* x, int32_t mem, foggy_stats* stats,
                        double* cross_sections);

/* y_v = A x_v for nrhs vectors one after the other (reference layout, foggy_vector_length entries
 * each): lib_mie_ms_solver_calculate_vector_b (lib_mie_ms_solver_interface.f90:739-783) for several
 * vectors in one call; each y_v equals foggy_matvec of x_v. */
int32_t foggy_matvec_rhs(foggy_handle h, int32_t nrhs, const double* x, double* y, int32_t mem);

/* ---- several right-hand sides in one block -------------------------------------------- */

/* The right-hand sides of one scene (one per plane wave set on the handle, nrhs = that count; no
 * Gaussian beams) solved together.  The reference solves each illumination with its own GMRES run
 * (lib_mie_ms_solver_run, lib_mie_ms_solver_interface.f90:143-154, around lib_solver_GMRES.f90:116-316);
 * here every operator application serves the whole block: each CTA of the operator applies the
 * translations of one target sphere to a tile of right-hand sides, whose width the library picks per
 * launch shape by timing (foggy_block_tiles); with matvec_mode = FOGGY_MATVEC_MLFMM the passes run
 * vector after vector inside each block application.  Each right-hand side keeps its own GMRES(m) recurrence
 * (gmres_restart 1..63, gmres_tolerance, gmres_max_iterations apply to each) and leaves the block when
 * its true residual meets the tolerance at a restart.  With params.precision = 1 the Arnoldi steps
 * apply the operator with FP32 translation arithmetic and the restart residuals in FP64.  x (and x0, if
 * not NULL) hold nrhs vectors of foggy_vector_length entries one after the other; cross_sections
 * ({C_sca, C_ext, C_abs} per right-hand side), iterations and backward_errors (per right-hand side) may
 * be NULL.  stats: iterations summed over right-hand sides, matvecs = vectors the operator was applied
 * to, the largest backward error; the status is that of the first right-hand side that failed. */
int32_t foggy_solve_block(foggy_handle h, int32_t nrhs, const double* x0, double* x, int32_t mem, foggy_stats* stats,
                          double* cross_sections, int32_t* iterations, double* backward_errors);

/* y_v = A x_v for nrhs vectors in one block operator application (the direct operator,
 * lib_mie_ms_solver_calculate_vector_b, lib_mie_ms_solver_interface.f90:739-783, applied to several
 * vectors at once; the ML-FMM passes vector after vector); precision 0 = FP64 translations, 1 = FP32
 * translations (FP64 vectors). */
int32_t foggy_matvec_block(foggy_handle h, int32_t nrhs, int32_t precision, const double* x, double* y, int32_t mem);

/* The block operator's tile width per launch for a block of nrhs vectors, tuned on first use:
 * out[4 i + 0..3] = (target spheres, source spheres, largest degree, right-hand sides per CTA) of
 * launch i.  out = NULL queries the launch count.  No counterpart in the reference. */
int32_t foggy_block_tiles(foggy_handle h, int32_t precision, int32_t nrhs, int32_t* out, int32_t* count);

/* ---- serving ------------------------------------------------------------------------- */

/* A solve server on one GPU: requests of differing sphere counts, truncation orders and
 * right-hand-side counts are queued first in, first out and admitted when their device footprint
 * (scene, operator slabs, Krylov workspace, staging and, when they fit an equal share of the
 * budget, pair tables) fits beside the requests already running; up to max_concurrent run at
 * once, each on its own handle and CUDA stream, so each result equals the one its request gets
 * alone.  A request larger than the whole budget is refused (FOGGY_REQ_REFUSED,
 * FOGGY_ERR_NOMEM).  memory_budget <= 0 takes 85 % of the free device memory.  The reference has
 * no serving layer; each request runs lib_mie_ms_solver_run with the direct operator. */
typedef struct foggy_server_s* foggy_server;

#define FOGGY_REQ_QUEUED    0
#define FOGGY_REQ_RUNNING   1
#define FOGGY_REQ_DONE      2
#define FOGGY_REQ_FAILED    3
#define FOGGY_REQ_CANCELLED 4
#define FOGGY_REQ_REFUSED   5

/* One request; every array is copied at submission (layouts as foggy_set_spheres and
 * foggy_set_plane_waves; phase and d_0_i may be NULL).  rhs_per_wave = 1 solves one right-hand
 * side per plane wave (foggy_solve_rhs), 0 one right-hand side of all waves together. */
typedef struct foggy_request {
    const foggy_params* params;
    int32_t n_spheres;
    const double* centres;
    const int32_t* param_index;
    int32_t n_param;
    const double* refractive_index;
    const double* radius;
    const int32_t* n_range;
    int32_t nw;
    const double* theta;
    const double* phi;
    const double* jones;
    const double* g;
    const double* phase;
    const double* d_0_i;
    int32_t rhs_per_wave;
} foggy_request;

typedef struct foggy_request_info {
    int32_t state;               /* FOGGY_REQ_*                                              */
    int32_t status;              /* FOGGY_OK or the solve's error                            */
    int32_t nrhs;
    int32_t reserved;
    int64_t x_len;               /* doubles in the result: nrhs vectors, 2 per complex entry  */
    int64_t footprint;           /* device bytes the request was admitted with               */
    double  ms_queued;           /* submission to start (or to now / to the end if it never ran) */
    double  ms_solve;            /* start to end                                             */
    double  ms_latency;          /* submission to end (or to now)                            */
    foggy_stats stats;
    char    error[256];
} foggy_request_info;

int32_t foggy_server_start(int32_t device, int32_t max_concurrent, int64_t memory_budget, foggy_server* out);
int32_t foggy_server_submit(foggy_server s, const foggy_request* request, int64_t* id);
/* State of a request; wait_ms > 0 waits up to that long for it to finish, < 0 without limit.
 * status, nrhs, x_len, stats and error are filled once the request has finished (zero before).
 * When it is done, copies the solutions into x (x_len doubles at least; NULL to skip) and the
 * cross-sections into cross_sections (3 nrhs doubles; NULL to skip). */
int32_t foggy_server_poll(foggy_server s, int64_t id, int32_t wait_ms, foggy_request_info* info, double* x,
                          int64_t x_len, double* cross_sections);
/* Removes a queued request (FOGGY_ERR_STATE once it runs). */
int32_t foggy_server_cancel(foggy_server s, int64_t id);
/* Frees a finished request's results. */
int32_t foggy_server_release(foggy_server s, int64_t id);
/* Cancels the queued requests, waits for the running ones and frees the server. */
int32_t foggy_server_stop(foggy_server s);

#ifdef __cplusplus
}
#endif

#endif /* FOGGY_GPU_H */
