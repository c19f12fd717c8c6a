"""Host-side mirror of the reference's multi-sphere solver interface.

The reference drives the solve through module-global Fortran state and these routines:
  lib_mie_ms_constructor                           FoggySim/src/lib/mie_theory/lib_mie_multi_sphere.f90:111-150
  lib_mie_ms_calculate_scattering_coefficients_ab_nm                             :162-371
  lib_mie_ms_solver_run / _use_ml_fmm / _set_n_range / _set_max_iterations /
  _get_backward_error                       lib_mie_ms_solver_interface.f90:143-209
  lib_mie_ms_solver_calculate_vector_b (the matvec)                              :739-783
  lib_mie_ms_solver_get_vector_b_all (the right-hand side)                       :230-315
  lib_math_vector_spherical_harmonics_translation_coefficient
                                   libmath/src/math/lib_math_vector_spherical_harmonics.f90:48-52
  lib_math_wigner_3j                                    libmath/src/math/lib_math_wigner.f90:45-72
  lib_tree_constructor / lib_tree_hf_get_universal_index            libtree/src/lib/lib_tree.f90:147-270
Here one MultiSphereSolver object holds that state and calls the C ABI of libfoggy_b200.so; all
arithmetic runs on the GPU.  Vectors use the reference's flat layout (complex128, per sphere
[a_nm | b_nm], n = 1..n_max, m = -n..n).
"""
import ctypes as C

import numpy as np

from . import _native as N


def _params(scene, use_ml_fmm=False, init_with_single_sphere=False, memory_budget=0, pair_tables=0,
            fmm_convention=0, z_translation_gt_r=3, precision=0, fmm_digits=0.0):
    L = N.load()
    p = N.FoggyParams()
    L.foggy_default_params(C.byref(p))
    p.lambda_0 = scene.lambda_0
    p.n_medium = scene.n_medium
    p.n_range[0] = int(scene.n_range[0])
    p.n_range[1] = int(scene.n_range[1])
    p.z_coupling = int(scene.z_coupling)
    p.reference_row_rule = int(bool(scene.reference_row_rule))
    p.matvec_mode = N.FOGGY_MATVEC_MLFMM if use_ml_fmm else N.FOGGY_MATVEC_DIRECT
    p.use_initial_guess = int(bool(init_with_single_sphere))
    p.gmres_restart = int(scene.gmres_restart)
    p.gmres_max_iterations = int(scene.gmres_max_iterations)
    p.gmres_tolerance = float(scene.gmres_tolerance)
    p.tree_l_max = int(scene.tree_l_max)
    p.device_memory_budget = int(memory_budget)
    p.pair_tables = int(pair_tables)
    p.fmm_convention = int(fmm_convention)
    p.z_translation_gt_r = int(z_translation_gt_r)
    p.precision = int(precision)
    p.fmm_digits = float(fmm_digits)
    return p


class MultiSphereSolver:
    """lib_mie_ms_constructor + the solver interface, on one GPU."""

    def __init__(self, scene, use_ml_fmm=False, init_with_single_sphere=False, device=0, memory_budget=0,
                 pair_tables=0, fmm_convention=0, z_translation_gt_r=3, precision=0, fmm_digits=0.0):
        """fmm_convention 0 runs the ML-FMM as the reference writes it, 1 the consistent
        expansion (see foggy_params.fmm_convention); fmm_digits > 0 expands each level's boxes to
        the excess-bandwidth order of that many digits instead of the global order."""
        self.L = N.load()
        self.scene = scene
        self.params = _params(scene, use_ml_fmm, init_with_single_sphere, memory_budget, pair_tables,
                              fmm_convention, z_translation_gt_r, precision, fmm_digits)
        h = C.c_void_p()
        N.check(self.L.foggy_create(C.byref(self.params), int(device), C.byref(h)))
        self.h = h
        s = scene
        self._keep = [N.as_f64(s.centres).reshape(-1), N.as_i32(s.param_index),
                      N.as_c128(s.refractive_index), N.as_f64(s.radius),
                      N.as_i32(s.n_range_param).reshape(-1)]
        c, pi, m, r, nr = self._keep
        N.check(self.L.foggy_set_spheres(self.h, s.n_spheres, N.ptr(c), N.ptr(pi, C.c_int32), s.n_param,
                                         N.ptr(m), N.ptr(r), N.ptr(nr, C.c_int32)), self.h)
        w = [N.as_f64(s.wave_theta), N.as_f64(s.wave_phi), N.as_f64(s.jones).reshape(-1),
             N.as_f64(s.wave_g), N.as_f64(s.wave_phase), N.as_f64(s.wave_d0).reshape(-1)]
        N.check(self.L.foggy_set_plane_waves(self.h, s.n_waves, *[N.ptr(a) for a in w]), self.h)
        self.n = int(self.L.foggy_vector_length(self.h))
        self.last_stats = None

    # ---- lifecycle --------------------------------------------------------------------
    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.L.foggy_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _set(self):
        N.check(self.L.foggy_set_params(self.h, C.byref(self.params)), self.h)

    # ---- lib_mie_ms_solver_* setters ------------------------------------------------------
    def use_ml_fmm(self, flag):
        self.params.matvec_mode = N.FOGGY_MATVEC_MLFMM if flag else N.FOGGY_MATVEC_DIRECT
        self._set()

    def set_max_iterations(self, it):
        self.params.gmres_max_iterations = int(it)
        self._set()

    def set_tolerance(self, tol):
        self.params.gmres_tolerance = float(tol)
        self._set()

    def set_restart(self, m):
        self.params.gmres_restart = int(m)
        self._set()

    def get_backward_error(self):
        return float(self.L.foggy_get_backward_error(self.h))

    # ---- building blocks ----------------------------------------------------------------
    def mie_coefficients(self, ip):
        p = int(min(self.scene.n_range_param[ip][1], self.scene.n_range[1]))
        a = np.zeros(p, np.complex128)
        b = np.zeros(p, np.complex128)
        N.check(self.L.foggy_get_mie_coefficients(self.h, int(ip), N.ptr(a), N.ptr(b)), self.h)
        return a, b

    def get_vector_b(self):
        b = np.zeros(self.n, np.complex128)
        N.check(self.L.foggy_get_vector_b(self.h, b.ctypes.data, N.FOGGY_MEM_HOST), self.h)
        return b

    def calculate_vector_b(self, x):
        """The operator y = A x (lib_mie_ms_solver_calculate_vector_b)."""
        x = N.as_c128(x)
        if x.size != self.n:
            raise ValueError("x has %d entries, expected %d" % (x.size, self.n))
        y = np.zeros(self.n, np.complex128)
        N.check(self.L.foggy_matvec(self.h, x.ctypes.data, y.ctypes.data, N.FOGGY_MEM_HOST), self.h)
        return y

    def matvec_device(self, x_ptr, y_ptr):
        """Operator on device buffers (reference layout) given as raw CUDA pointers."""
        N.check(self.L.foggy_matvec(self.h, C.c_void_p(x_ptr), C.c_void_p(y_ptr), N.FOGGY_MEM_DEVICE), self.h)

    # ---- the solve ------------------------------------------------------------------------
    def solve(self, x0=None, raise_on_error=True):
        """lib_mie_ms_solver_run: GMRES on the device; returns (x, stats)."""
        x = np.zeros(self.n, np.complex128)
        st = N.FoggyStats()
        x0p = None
        if x0 is not None:
            x0 = N.as_c128(x0)
            x0p = x0.ctypes.data
        rc = self.L.foggy_solve(self.h, x0p, x.ctypes.data, N.FOGGY_MEM_HOST, C.byref(st))
        self.last_stats = st.as_dict()
        if raise_on_error:
            N.check(rc, self.h)
        return x, self.last_stats

    def calculate_vector_b_rhs(self, X):
        """y_v = A x_v for the rows of X (foggy_matvec_rhs)."""
        X = N.as_c128(np.asarray(X).reshape(-1))
        nr = X.size // self.n
        Y = np.zeros(nr * self.n, np.complex128)
        N.check(self.L.foggy_matvec_rhs(self.h, nr, X.ctypes.data, Y.ctypes.data, N.FOGGY_MEM_HOST), self.h)
        return Y.reshape(nr, self.n)

    def solve_rhs(self, x0=None, raise_on_error=True):
        """One solve per plane wave (foggy_solve_rhs): x of shape (nrhs, n), cross-sections
        (nrhs, 3) as {C_sca, C_ext, C_abs}, summed stats."""
        nrhs = self.scene.n_waves
        x = np.zeros(nrhs * self.n, np.complex128)
        cs = np.zeros(3 * nrhs)
        st = N.FoggyStats()
        x0p = None
        if x0 is not None:
            x0 = N.as_c128(np.asarray(x0).reshape(-1))
            x0p = x0.ctypes.data
        rc = self.L.foggy_solve_rhs(self.h, nrhs, x0p, x.ctypes.data, N.FOGGY_MEM_HOST, C.byref(st), cs.ctypes.data)
        self.last_stats = st.as_dict()
        if raise_on_error:
            N.check(rc, self.h)
        return x.reshape(nrhs, self.n), cs.reshape(nrhs, 3), self.last_stats

    def solve_block(self, x0=None, raise_on_error=True):
        """All plane waves' right-hand sides in one block (foggy_solve_block): x of shape (nrhs, n),
        cross-sections (nrhs, 3), per-right-hand-side iterations and backward errors, summed stats."""
        nrhs = self.scene.n_waves
        x = np.zeros(nrhs * self.n, np.complex128)
        cs = np.zeros(3 * nrhs)
        its = np.zeros(nrhs, np.int32)
        be = np.zeros(nrhs)
        st = N.FoggyStats()
        x0p = None
        if x0 is not None:
            x0 = N.as_c128(np.asarray(x0).reshape(-1))
            x0p = x0.ctypes.data
        rc = self.L.foggy_solve_block(self.h, nrhs, x0p, x.ctypes.data, N.FOGGY_MEM_HOST, C.byref(st), cs.ctypes.data,
                                      its.ctypes.data, be.ctypes.data)
        self.last_stats = st.as_dict()
        if raise_on_error:
            N.check(rc, self.h)
        return x.reshape(nrhs, self.n), cs.reshape(nrhs, 3), its, be, self.last_stats

    def calculate_vector_b_block(self, X, precision=0):
        """y_v = A x_v for the rows of X in one block application (foggy_matvec_block); precision 1
        uses FP32 translation arithmetic."""
        X = N.as_c128(np.asarray(X).reshape(-1))
        nr = X.size // self.n
        Y = np.zeros(nr * self.n, np.complex128)
        N.check(self.L.foggy_matvec_block(self.h, nr, int(precision), X.ctypes.data, Y.ctypes.data,
                                          N.FOGGY_MEM_HOST), self.h)
        return Y.reshape(nr, self.n)

    def block_tiles(self, nrhs, precision=0):
        """(targets, sources, largest degree, right-hand sides per CTA) of each operator launch."""
        cnt = C.c_int32(0)
        N.check(self.L.foggy_block_tiles(self.h, int(precision), int(nrhs), None, C.byref(cnt)), self.h)
        out = np.zeros(4 * cnt.value, np.int32)
        N.check(self.L.foggy_block_tiles(self.h, int(precision), int(nrhs), N.ptr(out, C.c_int32), C.byref(cnt)),
                self.h)
        return out.reshape(-1, 4)

    def solve_device(self, x_ptr, x0_ptr=None):
        st = N.FoggyStats()
        rc = self.L.foggy_solve(self.h, C.c_void_p(x0_ptr) if x0_ptr else None, C.c_void_p(x_ptr),
                                N.FOGGY_MEM_DEVICE, C.byref(st))
        self.last_stats = st.as_dict()
        N.check(rc, self.h)
        return self.last_stats

    def set_n_range(self, n_range):
        """lib_mie_ms_solver_set_n_range (lib_mie_ms_solver_interface.f90:174-189): the global degree
        range; each sphere is truncated at the smaller of its own and the global n_max."""
        self.params.n_range[0] = int(n_range[0])
        self.params.n_range[1] = int(n_range[1])
        self._set()
        self.n = int(self.L.foggy_vector_length(self.h))

    def set_gaussian_beams(self, waist, tem, theta, phi, jones, g, phase=None, d_0_i=None, convention=None):
        """Gaussian beams added to the plane waves (foggy_set_gaussian_beams; the reference's
        lib_mie_illumination_gaussian_beam_parameter list with calculation_type 3).  waist (nb, 2),
        tem (nb, 2), theta, phi, g, phase (nb,), jones (nb, 4) re x, im x, re y, im y,
        d_0_i (nb, 3), convention (nb,)."""
        nb = len(np.atleast_1d(theta))
        arrs = [N.as_f64(waist).reshape(-1), N.as_i32(tem).reshape(-1), N.as_f64(theta), N.as_f64(phi),
                N.as_f64(jones).reshape(-1), N.as_f64(g),
                N.as_f64(phase) if phase is not None else None,
                N.as_f64(d_0_i).reshape(-1) if d_0_i is not None else None,
                N.as_i32(convention) if convention is not None else None]
        self._beams = arrs
        ptrs = [(a.ctypes.data if a is not None else None) for a in arrs]
        N.check(self.L.foggy_set_gaussian_beams(self.h, nb, *ptrs), self.h)

    def set_plane_waves(self, theta, phi, jones, g, phase, d_0_i):
        """Replace the plane waves (an empty list leaves only the Gaussian beams)."""
        w = [N.as_f64(theta), N.as_f64(phi), N.as_f64(jones).reshape(-1), N.as_f64(g), N.as_f64(phase),
             N.as_f64(d_0_i).reshape(-1)]
        self._waves = w
        N.check(self.L.foggy_set_plane_waves(self.h, len(w[0]), *[N.ptr(a) for a in w]), self.h)

    def n_range(self):
        return int(self.params.n_range[0]), int(self.params.n_range[1])

    @staticmethod
    def embed(x, n_spheres, n_from, n_to):
        """Coefficients of degree range (1, n_from) in the layout of (1, n_to): common degrees
        copied, the rest zero, as lib_mie_ms_solver_get_vector_x_all rebuilds the initial guess
        from the stored per-sphere a_nm, b_nm (lib_mie_ms_solver_interface.f90:467-520)."""
        cf = (n_from + 1) ** 2 - 1
        ct = (n_to + 1) ** 2 - 1
        cm = min(cf, ct)
        src = np.asarray(x).reshape(n_spheres, 2, cf)
        out = np.zeros((n_spheres, 2, ct), np.complex128)
        out[:, :, :cm] = src[:, :, :cm]
        return out.reshape(-1)

    def calculate_scattering_coefficients_ab_nm(self, update_initial_guess_with_n_max=None, step_size=None,
                                                dynamic_step_size=False):
        """lib_mie_ms_calculate_scattering_coefficients_ab_nm
        (FoggySim/src/lib/mie_theory/lib_mie_multi_sphere.f90:162-371): solve, optionally first at a
        lower n_max whose solution seeds the next solve (n_max continuation), and split the solution
        into per-sphere a_nm, b_nm arrays (n = 1..n_max, m = -n..n flattened).  Each stage's
        solution is the next stage's initial guess when the handle uses initial guesses (the
        reference stores every run's solution in its sphere list and reads it back only then).
        The stages run are listed in self.continuation_log as dicts (n_max, max_iterations,
        iterations, backward_error)."""
        n_org = self.n_range()
        max_it_org = int(self.params.gmres_max_iterations)
        state = {"x": None, "n": None}
        self.continuation_log = []

        def run(n_max, max_iterations):
            if n_max != self.n_range()[1]:
                self.set_n_range((n_org[0], n_max))
            if max_iterations is not None:
                self.set_max_iterations(max_iterations)
            x0 = None
            if self.params.use_initial_guess and state["x"] is not None:
                x0 = self.embed(state["x"], self.scene.n_spheres, state["n"], n_max)
            x, st = self.solve(x0, raise_on_error=False)
            state["x"], state["n"] = x, n_max
            self.continuation_log.append(dict(n_max=n_max, max_iterations=int(self.params.gmres_max_iterations),
                                              iterations=st["iterations"], backward_error=st["backward_error"]))
            return st["backward_error"]

        try:
            continuation_stages(run, n_org[1], update_initial_guess_with_n_max, step_size, dynamic_step_size)
        finally:
            if self.n_range() != n_org:
                self.set_n_range(n_org)
            self.set_max_iterations(max_it_org)
        st = self.last_stats
        if st["status"] != 0:
            N.check(st["status"], self.h)
        return self.split(state["x"]), st

    def split(self, x):
        c = (self.scene.n_range[1] + 1) ** 2 - 1
        x = np.asarray(x).reshape(self.scene.n_spheres, 2, c)
        return x[:, 0, :], x[:, 1, :]

    def cross_sections(self, x):
        """{C_sca, C_ext, C_abs} of the whole cluster for coefficient vector x."""
        x = N.as_c128(x)
        out = np.zeros(3)
        N.check(self.L.foggy_cross_sections(self.h, x.ctypes.data, N.FOGGY_MEM_HOST, N.ptr(out)), self.h)
        return out

    def get_field(self, x, points, e_field_0=1.0):
        """Scattered E and H (complex, shape (npoints, 3), cartesian) of coefficients x at points
        (lib_mie_ms_get_field); zero inside a sphere."""
        x = N.as_c128(x)
        pts = N.as_f64(points).reshape(-1)
        npt = len(pts) // 3
        E = np.zeros(3 * npt, np.complex128)
        H = np.zeros(3 * npt, np.complex128)
        N.check(self.L.foggy_get_field(self.h, x.ctypes.data, N.FOGGY_MEM_HOST, npt, pts.ctypes.data,
                                       float(e_field_0), E.ctypes.data, H.ctypes.data), self.h)
        return E.reshape(npt, 3), H.reshape(npt, 3)

    # ---- libtree -----------------------------------------------------------------------
    def build_tree(self):
        n = self.scene.n_spheres
        u = np.zeros(n, np.int64)
        order = np.zeros(n, np.int32)
        lmin = C.c_int32()
        lmax = C.c_int32()
        N.check(self.L.foggy_build_tree(self.h, N.ptr(u, C.c_int64), N.ptr(order, C.c_int32), C.byref(lmin),
                                        C.byref(lmax)), self.h)
        return u, order, lmin.value, lmax.value

    def tree_domain(self, level, n, kind):
        """E1 (kind 1) / E2 (kind 2) sphere lists or the I4 (kind 4) box list of box n at a level
        (lib_tree_get_domain_e1 / _e2 / _i4)."""
        cnt = C.c_int32(0)
        N.check(self.L.foggy_tree_domain(self.h, int(level), int(n), int(kind), None, C.byref(cnt)), self.h)
        out = np.zeros(max(cnt.value, 1), np.int64)
        N.check(self.L.foggy_tree_domain(self.h, int(level), int(n), int(kind), N.ptr(out, C.c_int64), C.byref(cnt)),
                self.h)
        return out[:cnt.value]

    def tree_boxes(self, level):
        cnt = C.c_int32(0)
        N.check(self.L.foggy_tree_boxes(self.h, int(level), None, C.byref(cnt)), self.h)
        out = np.zeros(cnt.value, np.int64)
        N.check(self.L.foggy_tree_boxes(self.h, int(level), N.ptr(out, C.c_int64), C.byref(cnt)), self.h)
        return out


# ---- libmath / libtree free functions ---------------------------------------------------------
def translation_coefficient(x, theta, phi, n_range, nu_range, z_selector):
    """A_mn^{mu nu}, B_mn^{mu nu} (reference layout, rows (n, m), columns (nu, mu))."""
    L = N.load()
    cn = (n_range[1] + 1) ** 2 - n_range[0] ** 2
    cnu = (nu_range[1] + 1) ** 2 - nu_range[0] ** 2
    A = np.zeros((cn, cnu), np.complex128)
    B = np.zeros((cn, cnu), np.complex128)
    nr = (C.c_int32 * 2)(*n_range)
    nur = (C.c_int32 * 2)(*nu_range)
    N.check(L.foggy_translation_coefficients(float(x), float(theta), float(phi), nr, nur, int(z_selector),
                                             N.ptr(A), N.ptr(B)))
    return A, B


def wigner_3j(j1, j2, j3, m1, m2, m3):
    return float(N.load().foggy_wigner_3j(j1, j2, j3, m1, m2, m3))


def universal_index(points, level):
    pts = N.as_f64(points).reshape(-1)
    out = np.zeros(len(pts) // 3, np.int64)
    N.check(N.load().foggy_universal_index(len(out), N.ptr(pts), int(level), N.ptr(out, C.c_int64)))
    return out


def estimate_solve_bytes(scene, precision=0, use_ml_fmm=False, fmm_digits=0.0):
    """(solve bytes, pair-table bytes) a solve of scene holds on the device at its peak
    (foggy_estimate_solve_bytes; host only, no GPU); use_ml_fmm adds the ML-FMM's buffers."""
    p = _params(scene, use_ml_fmm=use_ml_fmm, precision=precision, fmm_digits=fmm_digits)
    sb, tb = C.c_int64(), C.c_int64()
    N.check(N.load().foggy_estimate_solve_bytes(C.byref(p), scene.n_spheres, N.ptr(N.as_i32(scene.param_index), C.c_int32),
                                               scene.n_param, N.ptr(N.as_i32(scene.n_range_param).reshape(-1), C.c_int32),
                                               C.byref(sb), C.byref(tb)))
    return sb.value, tb.value


def tree_parent(n, level, step=1):
    """lib_tree_get_parent (libtree/src/lib/lib_tree.f90:405-431): the box `step` levels above box
    n of the given level."""
    out = C.c_int64()
    N.check(N.load().foggy_tree_parent(int(n), int(level), int(step), C.byref(out)))
    return out.value


def tree_children(n, level):
    """lib_tree_get_children (lib_tree.f90:444-453): the eight boxes of level + 1 inside box n."""
    out = np.zeros(8, np.int64)
    N.check(N.load().foggy_tree_children(int(n), int(level), N.ptr(out, C.c_int64)))
    return out


def tree_centre_of_box(n, level):
    """lib_tree_get_centre_of_box (lib_tree.f90:1292-1300): centre of box n in the normalised cube."""
    out = np.zeros(3)
    N.check(N.load().foggy_tree_centre_of_box(int(n), int(level), N.ptr(out)))
    return out


def tree_neighbours(n, level):
    """lib_tree_hf_get_neighbour_all_xD with k = 1 (libtree/src/lib/lib_tree_helper_functions.f90:914-997):
    the boxes at distance 1 inside the domain, ascending."""
    out = np.zeros(26, np.int64)
    cnt = C.c_int32()
    N.check(N.load().foggy_tree_neighbours(int(n), int(level), N.ptr(out, C.c_int64), C.byref(cnt)))
    return out[:cnt.value]


def continuation_stages(run, n_org, n_start=None, step_size=None, dynamic=False):
    """The stage sequence of lib_mie_ms_calculate_scattering_coefficients_ab_nm
    (FoggySim/src/lib/mie_theory/lib_mie_multi_sphere.f90:162-371) over run(n_max, max_iterations)
    -> backward error (max_iterations None keeps the current setting):
      no n_start            one solve at n_org;
      n_start, no step      n_start with 100 iterations, then n_org with 1000;
      n_start, step         n_start, n_start + step, ... up to n_org - step with 100 each, then
                            n_org with 1000 (calc_with_steps, :238-266);
      n_start, step, dynamic  calc_with_dynmaic_step_size (:268-369): solve at n_start, then
                            repeatedly try the next degree with one iteration and accept the step
                            when the backward error stays below 1e-3, else halve it.  As in the
                            reference, an accepted trial (and every step of size 1) advances n_max
                            by the step a second time before the full solve, and a rejected trial
                            keeps the degree it tried."""
    if n_start is None:
        run(n_org, None)
        return
    if step_size is None:
        run(n_start, 100)
        run(n_org, 1000)
        return
    if not dynamic:
        for n in range(n_start, n_org - step_size + 1, step_size):
            run(n, 100)
        run(n_org, 1000)
        return
    m_step = step_size
    n = n_start
    run(n, None)
    state = "test"
    for _ in range(100000):
        if state == "test":
            n = n_org if n + m_step >= n_org else n + m_step
            if m_step > 1:
                berr = run(n, 1)
                if berr < 1e-3:
                    n = n_org if n + m_step >= n_org else n + m_step
                    state = "calculate"
                else:
                    state = "too_big" if m_step > 1 else "calculate"
            else:
                n = n_org if n + m_step >= n_org else n + m_step
                state = "calculate"
        elif state == "calculate":
            run(n, 1000)
            m_step = step_size
            state = "finish" if n == n_org else "test"
        elif state == "too_big":
            m_step = int(m_step / 2.0) if int(m_step / 2.0) > 1 else 1
            state = "test"
        else:
            return
    raise RuntimeError("continuation did not finish")
