"""Seeded synthetic scenes of the multi-sphere solve.

A Scene carries exactly the data the reference keeps in its module-global simulation_data
(FoggySim/src/lib/mie_theory/lib_mie_type.f90:43-99): the sphere list (centres, parameter index),
the shared sphere parameters (refractive index, radius, degree range), the global degree range,
the z-selector of the coupling and the plane waves; plus the GMRES settings.

Workloads (all lengths in micrometres, n_medium = 1, m = 1.33 + 1e-8 i, lambda = 0.55):
  small_cluster   64 spheres r = 0.5 in a 10 um cube, p = 15, GMRES(30) to 1e-8, 3 tree levels
  medium_cluster  2000 spheres, lognormal r (median 0.6, sigma_ln 0.3, clipped to 0.2..1.5) in a
                  40 um cube, per-sphere p by the Wiscombe rule, GMRES(50) to 1e-8, 5 levels
Centres are uniform in the cube with rejection of overlapping spheres.
"""
import dataclasses
import math

import numpy as np

M_WATER = complex(1.33, 1e-8)


def wiscombe_n_max(x):
    """n_max = ceil(x + 4 x^(1/3) + 2) (Wiscombe; the reference rounds up the same way,
    lib_mie_ss_helper_functions.f90:937-951, with 4.05 in place of 4)."""
    return int(math.ceil(x + 4.0 * x ** (1.0 / 3.0) + 2.0))


@dataclasses.dataclass
class Scene:
    lambda_0: float
    n_medium: float
    centres: np.ndarray          # (N, 3)
    param_index: np.ndarray      # (N,) int32, 0-based
    refractive_index: np.ndarray  # (NP,) complex
    radius: np.ndarray           # (NP,)
    n_range_param: np.ndarray    # (NP, 2) int32
    n_range: tuple               # global (1, n_max)
    wave_theta: np.ndarray
    wave_phi: np.ndarray
    jones: np.ndarray            # (nw, 4): re x, im x, re y, im y
    wave_g: np.ndarray
    wave_phase: np.ndarray
    wave_d0: np.ndarray          # (nw, 3)
    z_coupling: int = 3
    reference_row_rule: bool = False
    gmres_restart: int = 30
    gmres_tolerance: float = 1e-8
    gmres_max_iterations: int = 1000
    tree_l_max: int = 0
    name: str = "scene"

    @property
    def n_spheres(self):
        return int(self.centres.shape[0])

    @property
    def n_param(self):
        return int(self.radius.shape[0])

    @property
    def n_waves(self):
        return int(self.wave_theta.shape[0])

    @property
    def wavenumber(self):
        return 2.0 * math.pi * self.n_medium / self.lambda_0

    def p_of_sphere(self):
        p = np.minimum(self.n_range_param[:, 1], self.n_range[1])
        return p[self.param_index]

    def ragged_unknowns(self):
        p = self.p_of_sphere().astype(np.int64)
        return int(np.sum(2 * p * (p + 2)))

    def vector_length(self):
        c = (self.n_range[1] + 1) ** 2 - 1
        return 2 * c * self.n_spheres


def place_spheres(rng, radii, box):
    """Uniform centres in [0, box)^3, rejecting overlaps |c_i - c_j| < r_i + r_j."""
    n = len(radii)
    cell = 2.0 * float(np.max(radii))
    grid = {}
    centres = np.zeros((n, 3))
    for i in range(n):
        for _ in range(100000):
            c = rng.uniform(0.0, box, 3)
            key = tuple((c // cell).astype(int))
            ok = True
            for dx in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for dz in (-1, 0, 1):
                        for j in grid.get((key[0] + dx, key[1] + dy, key[2] + dz), ()):
                            if np.sum((centres[j] - c) ** 2) < (radii[i] + radii[j]) ** 2:
                                ok = False
                                break
                        if not ok:
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if ok:
                centres[i] = c
                grid.setdefault(key, []).append(i)
                break
        else:
            raise RuntimeError("could not place sphere %d" % i)
    return centres


def single_wave(theta=0.0, phi=0.0, jones=(1.0, 0.0, 0.0, 0.0)):
    """One plane wave; Jones (1, 0) along +z is the reference's x-polarised TM wave
    (lib_mie_type_functions.f90:156-158)."""
    return dict(wave_theta=np.array([theta]), wave_phi=np.array([phi]),
                jones=np.array([list(jones)], dtype=np.float64), wave_g=np.array([1.0]),
                wave_phase=np.array([0.0]), wave_d0=np.zeros((1, 3)))


def make_scene(radii, box, seed, lambda_0=0.55, n_medium=1.0, m=M_WATER, n_max=None, **kw):
    rng = np.random.default_rng(seed)
    radii = np.asarray(radii, dtype=np.float64)
    centres = place_spheres(rng, radii, box)
    k = 2.0 * math.pi * n_medium / lambda_0
    uniq, inv = np.unique(radii, return_inverse=True)
    p = np.array([wiscombe_n_max(k * r) if n_max is None else n_max for r in uniq], dtype=np.int32)
    nrp = np.stack([np.ones_like(p), p], axis=1).astype(np.int32)
    waves = kw.pop("waves", single_wave())
    return Scene(lambda_0=lambda_0, n_medium=n_medium, centres=centres,
                 param_index=inv.astype(np.int32), refractive_index=np.full(len(uniq), m, np.complex128),
                 radius=uniq, n_range_param=nrp, n_range=(1, int(p.max())), **waves, **kw)


def small_cluster(seed=1, z_coupling=3):
    """64 monodisperse water spheres, r = 0.5 um, 10 um cube, p = 15, GMRES(30) to 1e-8."""
    return make_scene(np.full(64, 0.5), 10.0, seed, z_coupling=z_coupling, reference_row_rule=True,
                      gmres_restart=30, gmres_tolerance=1e-8, tree_l_max=3, name="small_cluster_64")


def lognormal_radii(rng, n, median=0.6, sigma=0.3, lo=0.2, hi=1.5):
    return np.clip(median * np.exp(sigma * rng.standard_normal(n)), lo, hi)


def medium_cluster(seed=2, n=2000, box=40.0, z_coupling=3):
    """2000 lognormal water spheres in a 40 um cube, per-sphere Wiscombe p, GMRES(50) to 1e-8."""
    rng = np.random.default_rng(1000 + seed)
    radii = lognormal_radii(rng, n)
    return make_scene(radii, box, seed, z_coupling=z_coupling, reference_row_rule=False,
                      gmres_restart=50, gmres_tolerance=1e-8, tree_l_max=5,
                      name="medium_cluster_%d" % n)


def random_cluster(n, seed, p=None, box=None, radii=None, z_coupling=3, reference_row_rule=None,
                   waves=None, m=M_WATER):
    """Small polydisperse clusters for parity tests."""
    rng = np.random.default_rng(500 + seed)
    if radii is None:
        radii = rng.uniform(0.15, 0.45, n)
    if box is None:
        box = max(2.0, (n * 60.0) ** (1.0 / 3.0))
    kw = {}
    if waves is not None:
        kw["waves"] = waves
    sc = make_scene(radii, box, seed, n_max=p, m=m, z_coupling=z_coupling,
                    reference_row_rule=bool(reference_row_rule), **kw)
    return sc


# ---- hcp lattice scenes (FoggySim/src/lib/scene/lib_scene_generator.f90:53-280) -------------

def hcp_lattice(i, j, k, sphere_radius):
    """Centre of hcp site (i, j, k) for spheres of the given radius
    (lib_scene_gerator_hcp_lattice, lib_scene_generator.f90:53-67)."""
    x = 2.0 * i + math.fmod(float(j + k), 2.0)
    y = math.sqrt(3.0) * (j + math.fmod(float(k), 2.0) / 3.0)
    z = 2.0 * math.sqrt(6.0) * k / 3.0
    return np.array([x, y, z]) * sphere_radius


def hcp_fill_cuboid(size_x, size_y, size_z, sphere_radius):
    """hcp sites filling a cuboid, centred on the origin, in the reference's (i, j, k) order
    (lib_scene_generator_hcp_lattice_fill_cuboid, lib_scene_generator.f90:69-135)."""
    r = sphere_radius
    max_k = max(int(math.floor((size_z - 2.0 * r) / r * 3.0 / (2.0 * math.sqrt(6.0)))), 0)
    max_j = max(int(math.floor((size_y - 2.0 * r) / r / math.sqrt(3.0) - math.fmod(float(max_k), 2.0) / 3.0)), 0)
    max_i = max(int(math.floor(((size_x - 2.0 * r) / r - math.fmod(float(max_j + max_k), 2.0)) / 2.0)), 0)
    offset = -hcp_lattice(max_i, max_j, max_k, r) / 2.0
    out = np.empty(((max_i + 1) * (max_j + 1) * (max_k + 1), 3))
    x = 0
    for i in range(max_i + 1):
        for j in range(max_j + 1):
            for k in range(max_k + 1):
                out[x] = hcp_lattice(i, j, k, r) + offset
                x += 1
    return out


def hcp_fill_sphere(sphere_radius, lattice_sphere_radius, cap_plane_point=None, cap_plane_normal=None):
    """hcp sites inside a sphere (optionally the cap on the negative side of a plane), as the mask
    the reference keeps beside the cuboid lattice (lib_scene_generator_hcp_lattice_fill_sphere,
    lib_scene_generator.f90:137-203): a site is inside when |c| < R - r/2 and, with a cap plane,
    (c - point) . normal < 0 (the normal as given, not normalised, as the reference uses it)."""
    cub = hcp_fill_cuboid(2.0 * sphere_radius, 2.0 * sphere_radius, 2.0 * sphere_radius, lattice_sphere_radius)
    rho = np.sqrt(np.sum(cub * cub, axis=1))
    inside = rho < sphere_radius - lattice_sphere_radius / 2.0
    if cap_plane_point is not None and cap_plane_normal is not None:
        dist = (cub - np.asarray(cap_plane_point, np.float64)) @ np.asarray(cap_plane_normal, np.float64)
        inside &= dist < 0.0
    return cub, inside


def hcp_sphere_scene(sphere_radius, lattice_sphere_radius=0.0076, particle_radius=0.0075,
                     n_particle=complex(2.5287, 0.0), lambda_0=0.55):
    """The scene of the reference's hcp benchmark (lib_mie_ms_benchmark, calculate_sphere_scene,
    FoggySim/src/lib/mie_theory/lib_mie_multi_sphere.f90:3717-4164), in micrometres: particles of
    radius 7.5 nm, refractive index 2.5287, on an hcp lattice of 7.6 nm spheres filling the half
    (z < 0) of a sphere of the given radius; n_medium = 1, lambda = 550 nm; one plane wave along +z
    from (0, 0, -10 um), linear polarisation rotated by pi/4; z = j_n for the coupling.
    n_max = ceil(1.2 n_c) with the reference's n_c = ceil(x + 4.05 x^(1/3) + 2), the degree its
    convergence test (lib_mie_ss_test_convergence_plane_wave, lib_mie_single_sphere.f90:1604-1674)
    returns for these absolutely convergent Rayleigh-size series."""
    cub, inside = hcp_fill_sphere(sphere_radius, lattice_sphere_radius, (0.0, 0.0, 0.0), (0.0, 0.0, 1.0))
    centres = cub[inside]
    n_medium = 1.0
    x = 2.0 * math.pi * n_medium * particle_radius / lambda_0
    n_c = int(math.ceil(x + 4.05 * x ** (1.0 / 3.0) + 2.0))
    n_max = int(math.ceil(n_c * 1.2))
    c = math.cos(math.pi / 4.0)
    s = math.sin(math.pi / 4.0)
    waves = dict(wave_theta=np.array([0.0]), wave_phi=np.array([0.0]),
                 jones=np.array([[c, 0.0, s, 0.0]]), wave_g=np.array([1.0]),
                 wave_phase=np.array([0.0]), wave_d0=np.array([[0.0, 0.0, -10.0]]))
    n = len(centres)
    return Scene(lambda_0=lambda_0, n_medium=n_medium, centres=np.ascontiguousarray(centres),
                 param_index=np.zeros(n, np.int32), refractive_index=np.array([n_particle], np.complex128),
                 radius=np.array([particle_radius]), n_range_param=np.array([[1, n_max]], np.int32),
                 n_range=(1, n_max), z_coupling=1, reference_row_rule=True, gmres_restart=10,
                 gmres_tolerance=1e-6, name="hcp_sphere_%g" % sphere_radius, **waves)


# ---- serving stream ----------------------------------------------------------------------------

def serving_request(rng, n_lo=50, n_hi=500):
    """One request of the serving stream: sphere count log-uniform in [n_lo, n_hi], lognormal radii
    (median uniform in 0.4-0.8 um, sigma_ln 0.3, clipped to 0.2-1.2 um, orders up to 26, which
    keeps a 30-request stream within a few minutes), m = 1.33 + 1e-8 i, wavelength uniform in
    0.45-0.65 um, volume fraction uniform in 1-5 % (cube edge (N E[V] / vf)^(1/3)), 1-16
    right-hand sides along random directions, x-polarised (TM), GMRES(30) to 1e-6."""
    n = int(round(math.exp(rng.uniform(math.log(n_lo), math.log(n_hi)))))
    med = rng.uniform(0.4, 0.8)
    radii = np.clip(med * np.exp(0.3 * rng.standard_normal(n)), 0.2, 1.2)
    lam = rng.uniform(0.45, 0.65)
    vf = rng.uniform(0.01, 0.05)
    box = (np.sum(4.0 / 3.0 * math.pi * radii ** 3) / vf) ** (1.0 / 3.0)
    nr = int(rng.integers(1, 17))
    th = np.arccos(rng.uniform(-1.0, 1.0, nr))
    ph = rng.uniform(0.0, 2.0 * math.pi, nr)
    waves = dict(wave_theta=th, wave_phi=ph, jones=np.tile([1.0, 0.0, 0.0, 0.0], (nr, 1)), wave_g=np.ones(nr),
                 wave_phase=np.zeros(nr), wave_d0=np.zeros((nr, 3)))
    return make_scene(radii, box, int(rng.integers(1 << 30)), lambda_0=lam, waves=waves, z_coupling=3,
                      reference_row_rule=False, gmres_restart=30, gmres_tolerance=1e-6,
                      name="serving_%d" % n)
