"""ctypes wrapper of the FP64 CPU oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py import this module.
It loads oracle/liboracle.so, which restates the reference algorithms (see oracle.cpp) and
links the reference's own wigxjpf library built into oracle/_ref/.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
lp = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")


def build():
    """Compile liboracle.so (and _ref/libwigxjpf.a from the reference checkout named by the
    environment variable FOGGY_REFERENCE; without it the prebuilt _ref/ library is used)."""
    ref = os.environ.get("FOGGY_REFERENCE", "")
    args = ["make", "-s", "-C", HERE]
    if ref and os.path.isdir(ref):
        args.append("REF=" + ref)
    elif not os.path.exists(os.path.join(HERE, "_ref", "libwigxjpf.a")):
        raise RuntimeError("oracle/_ref/libwigxjpf.a is missing: set FOGGY_REFERENCE to the reference checkout")
    subprocess.run(args, check=True)


def lib():
    global _LIB
    if _LIB is not None:
        return _LIB
    path = os.path.join(HERE, "liboracle.so")
    if not os.path.exists(path):
        build()
    L = C.CDLL(path)
    L.orc_init.argtypes = [C.c_int]
    L.orc_sph_jn.argtypes = [C.c_double, C.c_int, dp]
    L.orc_sph_yn.argtypes = [C.c_double, C.c_int, dp]
    L.orc_legendre_table.argtypes = [C.c_double, C.c_int, dp]
    L.orc_pi_tau.argtypes = [C.c_double, C.c_int, C.c_int, dp, dp]
    L.orc_wigner_3j.argtypes = [C.c_int] * 6
    L.orc_wigner_3j.restype = C.c_double
    L.orc_ab_xu_cruzan.argtypes = [C.c_int] * 5 + [dp]
    L.orc_n_c.argtypes = [C.c_double]
    L.orc_mie_ab.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, dp, dp]
    L.orc_translation_xu.argtypes = [C.c_double] * 3 + [C.c_int] * 5 + [dp, dp]
    L.orc_universal_index.argtypes = [dp, C.c_int]
    L.orc_universal_index.restype = C.c_int64
    L.orc_coordinate_binary.argtypes = [C.c_double]
    L.orc_coordinate_binary.restype = C.c_uint64
    L.orc_scale_points.argtypes = [C.c_int, dp, dp]
    L.orc_build_tree.argtypes = [C.c_int, dp, C.c_int, C.c_int, lp, ip,
                                 C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.orc_problem_create.restype = C.c_void_p
    L.orc_problem_create.argtypes = [C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int,
                                     C.c_int, dp, ip, C.c_int, dp, dp, ip, C.c_int,
                                     dp, dp, dp, dp, dp, dp]
    L.orc_problem_destroy.argtypes = [C.c_void_p]
    L.orc_vector_length.argtypes = [C.c_void_p]
    L.orc_vector_length.restype = C.c_int64
    L.orc_mie_of_param.argtypes = [C.c_void_p, C.c_int, dp, dp]
    L.orc_vector_b.argtypes = [C.c_void_p, dp, dp]
    L.orc_matvec.argtypes = [C.c_void_p, dp, dp]
    L.orc_solve.argtypes = [C.c_void_p, dp, dp, C.c_int, C.c_double, C.c_int, C.c_void_p,
                            ip, C.POINTER(C.c_double)]
    L.orc_cross_sections.argtypes = [C.c_void_p, dp, dp]
    L.orc_init(64)
    _LIB = L
    return L


def _c(a):
    """complex128 array -> interleaved float64 view."""
    a = np.ascontiguousarray(a, dtype=np.complex128)
    return a.view(np.float64)


def sph_jn(x, nmax):
    out = np.zeros(nmax + 1)
    lib().orc_sph_jn(x, nmax, out)
    return out


def sph_yn(x, nmax):
    out = np.zeros(nmax + 1)
    lib().orc_sph_yn(x, nmax, out)
    return out


def legendre_table(x, nmax):
    out = np.zeros((nmax + 1) ** 2)
    lib().orc_legendre_table(x, nmax, out)
    return out


def pi_tau(theta, nmax, cs_phase=False):
    pi = np.zeros((nmax + 1) ** 2)
    tau = np.zeros((nmax + 1) ** 2)
    lib().orc_pi_tau(theta, nmax, int(cs_phase), pi, tau)
    return pi, tau


def wigner_3j(j1, j2, j3, m1, m2, m3):
    return lib().orc_wigner_3j(j1, j2, j3, m1, m2, m3)


def ab_xu_cruzan(m, n, mu, nu, p):
    out = np.zeros(2)
    lib().orc_ab_xu_cruzan(m, n, mu, nu, p, out)
    return out[0], out[1]


def n_c(x):
    return lib().orc_n_c(x)


def mie_ab(x, m, n1, n2):
    a = np.zeros(2 * (n2 - n1 + 1))
    b = np.zeros(2 * (n2 - n1 + 1))
    lib().orc_mie_ab(x, complex(m).real, complex(m).imag, n1, n2, a, b)
    return a.view(np.complex128), b.view(np.complex128)


def translation_xu(x, theta, phi, n_range, nu_range, z):
    cn = (n_range[1] + 1) ** 2 - n_range[0] ** 2
    cnu = (nu_range[1] + 1) ** 2 - nu_range[0] ** 2
    A = np.zeros(2 * cn * cnu)
    B = np.zeros(2 * cn * cnu)
    lib().orc_translation_xu(x, theta, phi, n_range[0], n_range[1], nu_range[0], nu_range[1],
                             z, A, B)
    return A.view(np.complex128).reshape(cn, cnu), B.view(np.complex128).reshape(cn, cnu)


def universal_index(point, l):
    return lib().orc_universal_index(np.ascontiguousarray(point, dtype=np.float64), l)


def coordinate_binary(f):
    return lib().orc_coordinate_binary(f)


def scale_points(centres):
    c = np.ascontiguousarray(centres, dtype=np.float64).reshape(-1)
    out = np.zeros_like(c)
    lib().orc_scale_points(len(c) // 3, c, out)
    return out.reshape(-1, 3)


def build_tree(centres, s=10, l_max=0):
    c = np.ascontiguousarray(centres, dtype=np.float64).reshape(-1)
    n = len(c) // 3
    u = np.zeros(n, np.int64)
    order = np.zeros(n, np.int32)
    lmin = C.c_int(0)
    lmax = C.c_int(0)
    lib().orc_build_tree(n, c, s, l_max, u, order, C.byref(lmin), C.byref(lmax))
    return u, order, lmin.value, lmax.value


class Problem:
    """The multi-sphere problem in the reference's data model (lib_mie_type.f90:43-99)."""

    def __init__(self, scene):
        L = lib()
        s = scene
        self.scene = s
        self.h = L.orc_problem_create(
            s.lambda_0, s.n_medium, s.n_range[0], s.n_range[1], s.z_coupling,
            int(s.reference_row_rule), s.n_spheres,
            np.ascontiguousarray(s.centres, np.float64).reshape(-1),
            np.ascontiguousarray(s.param_index, np.int32), s.n_param,
            _c(s.refractive_index), np.ascontiguousarray(s.radius, np.float64),
            np.ascontiguousarray(s.n_range_param, np.int32).reshape(-1), s.n_waves,
            np.ascontiguousarray(s.wave_theta, np.float64),
            np.ascontiguousarray(s.wave_phi, np.float64),
            np.ascontiguousarray(s.jones, np.float64).reshape(-1),
            np.ascontiguousarray(s.wave_g, np.float64),
            np.ascontiguousarray(s.wave_phase, np.float64),
            np.ascontiguousarray(s.wave_d0, np.float64).reshape(-1))
        self.n = L.orc_vector_length(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_problem_destroy(self.h)
            self.h = None

    def mie(self, ip):
        a0, a1 = self.scene.n_range_param[ip]
        a = np.zeros(2 * (a1 - a0 + 1))
        b = np.zeros(2 * (a1 - a0 + 1))
        lib().orc_mie_of_param(self.h, ip, a, b)
        return a.view(np.complex128), b.view(np.complex128)

    def vector_b(self, with_pq=False):
        b = np.zeros(2 * self.n)
        pq = np.zeros(2 * self.n)
        lib().orc_vector_b(self.h, b, pq)
        if with_pq:
            return b.view(np.complex128), pq.view(np.complex128)
        return b.view(np.complex128)

    def matvec(self, x):
        y = np.zeros(2 * self.n)
        lib().orc_matvec(self.h, _c(x), y)
        return y.view(np.complex128)

    def solve(self, b=None, x0=None, restart=30, tol=1e-8, maxit=1000, weights=None):
        if b is None:
            b = self.vector_b()
        x = np.array(x0 if x0 is not None else np.zeros(self.n), dtype=np.complex128)
        xf = _c(x).copy()
        info = np.zeros(4, np.int32)
        berr = C.c_double(0.0)
        w = None
        if weights is not None:
            w = np.ascontiguousarray(weights, np.float64)
        lib().orc_solve(self.h, _c(b), xf, restart, tol, maxit,
                        w.ctypes.data_as(C.c_void_p) if w is not None else None,
                        info, C.byref(berr))
        return xf.view(np.complex128), dict(iterations=int(info[0]), restarts=int(info[1]),
                                            matvecs=int(info[2]), status=int(info[3]),
                                            backward_error=berr.value)

    def cross_sections(self, x):
        out = np.zeros(3)
        lib().orc_cross_sections(self.h, _c(x), out)
        return out


def _matvec_rows(self, x, j0, j1, cache=True):
    """Operator rows of target spheres j0 <= j < j1 (other entries zero)."""
    L = lib()
    if not getattr(L, "_rows_sig", False):
        L.orc_matvec_rows.argtypes = [C.c_void_p, dp, C.c_int, C.c_int, C.c_int, dp]
        L._rows_sig = True
    y = np.zeros(2 * self.n)
    L.orc_matvec_rows(self.h, _c(x), int(j0), int(j1), int(bool(cache)), y)
    return y.view(np.complex128)


Problem.matvec_rows = _matvec_rows


def _pairs_apply(self, x, targets, sources):
    """Contributions of ordered pairs (targets[i] <- sources[i]) to the operator, every
    translation block recomputed as in the reference."""
    L = lib()
    if not getattr(L, "_pairs_sig", False):
        L.orc_pairs_apply.argtypes = [C.c_void_p, dp, C.c_int, ip, ip, dp]
        L._pairs_sig = True
    y = np.zeros(2 * self.n)
    t = np.ascontiguousarray(targets, np.int32)
    s = np.ascontiguousarray(sources, np.int32)
    L.orc_pairs_apply(self.h, _c(x), len(t), t, s, y)
    return y.view(np.complex128)


Problem.pairs_apply = _pairs_apply


def _fmm_matvec(self, x, l_max=0, s_opt=10, convention=0, z_gt_r=3, digits=0.0):
    """The reference's ML-FMM operator y = A x (convention 0, as the Fortran does it) or the
    consistent expansion (convention 1); l_max > 0 fixes the leaf level; digits > 0 expands each
    level's boxes to the excess-bandwidth order of that many digits (not in the reference, which
    uses its global order everywhere; digits = 0)."""
    L = lib()
    if not getattr(L, "_fmm_sig", False):
        L.orc_fmm_matvec.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, dp, dp]
        L._fmm_sig = True
    y = np.zeros(2 * self.n)
    L.orc_fmm_matvec(self.h, int(l_max), int(s_opt), int(convention), int(z_gt_r), float(digits), _c(x), y)
    return y.view(np.complex128)


Problem.fmm_matvec = _fmm_matvec


def tree_domain(centres, l_max, l, n, kind):
    """E1 (kind 1), E2 (kind 2) sphere lists or I4 (kind 4) box list of box n at level l."""
    L = lib()
    if not getattr(L, "_dom_sig", False):
        L.orc_tree_domain.argtypes = [C.c_int, dp, C.c_int, C.c_int, C.c_int64, C.c_int, C.c_void_p, C.c_int]
        L.orc_tree_domain.restype = C.c_int
        L._dom_sig = True
    c = np.ascontiguousarray(centres, np.float64).reshape(-1)
    cnt = L.orc_tree_domain(len(c) // 3, c, int(l_max), int(l), int(n), int(kind), None, 0)
    out = np.zeros(max(cnt, 1), np.int64)
    L.orc_tree_domain(len(c) // 3, c, int(l_max), int(l), int(n), int(kind), out.ctypes.data, cnt)
    return out[:cnt]


def vswf(theta, phi, r, k, nmax, z=3):
    """M_nm, N_nm (n = 1..nmax, m = -n..n) as complex arrays [(n, m), (rho, theta, phi)]."""
    L = lib()
    if not getattr(L, "_vswf_sig", False):
        L.orc_vswf.argtypes = [C.c_double] * 4 + [C.c_int, C.c_int, dp, dp]
        L._vswf_sig = True
    cnt = (nmax + 1) ** 2 - 1
    M = np.zeros(6 * cnt)
    N = np.zeros(6 * cnt)
    L.orc_vswf(theta, phi, r, k, nmax, z, M, N)
    return M.view(np.complex128).reshape(cnt, 3), N.view(np.complex128).reshape(cnt, 3)


def _field(self, x, points, e0=1.0):
    """Scattered E, H (complex, shape (npoints, 3)) of coefficients x (reference layout)."""
    L = lib()
    if not getattr(L, "_field_sig", False):
        L.orc_field.argtypes = [C.c_void_p, dp, C.c_int, dp, C.c_double, dp, dp]
        L._field_sig = True
    pts = np.ascontiguousarray(points, np.float64).reshape(-1)
    n = len(pts) // 3
    E = np.zeros(6 * n)
    H = np.zeros(6 * n)
    L.orc_field(self.h, _c(x), n, pts, float(e0), E, H)
    return E.view(np.complex128).reshape(n, 3), H.view(np.complex128).reshape(n, 3)


Problem.field = _field


def _set_gaussian_beams(self, waist, tem, theta, phi, jones, g, phase=None, d0=None, convention=None):
    """Gaussian beams of the problem (plane-wave approximation, the reference's calculation_type 3)."""
    L = lib()
    nb = len(theta)
    arr = lambda a, t=np.float64: np.ascontiguousarray(a, t).reshape(-1)
    w, tm, th, ph, jo, gg = arr(waist), arr(tem, np.int32), arr(theta), arr(phi), arr(jones), arr(g)
    pa = arr(phase) if phase is not None else np.zeros(nb)
    dd = arr(d0) if d0 is not None else np.zeros(3 * nb)
    cv = arr(convention, np.int32) if convention is not None else np.ones(nb, np.int32)
    self._beams = (w, tm, th, ph, jo, gg, pa, dd, cv)
    L.orc_set_gaussian_beams(C.c_void_p(self.h), int(nb), w.ctypes.data_as(C.c_void_p),
                             tm.ctypes.data_as(C.c_void_p), th.ctypes.data_as(C.c_void_p),
                             ph.ctypes.data_as(C.c_void_p), jo.ctypes.data_as(C.c_void_p),
                             gg.ctypes.data_as(C.c_void_p), pa.ctypes.data_as(C.c_void_p),
                             dd.ctypes.data_as(C.c_void_p), cv.ctypes.data_as(C.c_void_p))


Problem.set_gaussian_beams = _set_gaussian_beams


def gaussian_probe(lambda0, n_medium, waist, tem, jones, theta, phi, phase, convention, points):
    """One Gaussian beam at points (beam origin at 0): scalar field (beam frame), (|E|, arg E) and
    the local plane wave (theta, phi, Jones x re/im, y re/im, phase, amplitude) per point."""
    L = lib()
    pts = np.ascontiguousarray(points, np.float64).reshape(-1)
    n = len(pts) // 3
    sc = np.zeros(2 * n)
    aa = np.zeros(2 * n)
    wv = np.zeros(8 * n)
    jo = np.ascontiguousarray(jones, np.float64)
    L.orc_gaussian_probe(C.c_double(lambda0), C.c_double(n_medium), C.c_double(waist[0]), C.c_double(waist[1]),
                         C.c_int(tem[0]), C.c_int(tem[1]), jo.ctypes.data_as(C.c_void_p), C.c_double(theta),
                         C.c_double(phi), C.c_double(phase), C.c_int(convention), C.c_int(n),
                         pts.ctypes.data_as(C.c_void_p), sc.ctypes.data_as(C.c_void_p),
                         aa.ctypes.data_as(C.c_void_p), wv.ctypes.data_as(C.c_void_p))
    return sc.view(np.complex128), aa.reshape(n, 2), wv.reshape(n, 8)
