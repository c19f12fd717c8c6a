"""hcp scene generator (FoggySim/src/lib/scene/lib_scene_generator.f90:53-280), the incident
plane-wave field and the field export (lib_field.f90:35-260, libtoolbox/src/file_io.f90) on the CPU."""
import math
import os

import numpy as np
import pytest

from itofoggysim_b200 import fields, hcp_benchmark, scene as S


def test_rot_matrix_reference_golden():
    # test_lib_math_get_matrix_rot (libmath/src/math/lib_math_type_operator.f90:6439-6520)
    R = fields.rot_matrix(math.pi / 2, math.pi / 2, math.pi / 2)
    for v, ref in [((1, 0, 0), (0, 0, 1)), ((0, 1, 0), (0, -1, 0)), ((0, 0, 1), (1, 0, 0))]:
        assert np.allclose(R @ np.array(v, float), ref, atol=1e-15)
    R = fields.rot_matrix(0.3, 1.1, -0.7)
    assert np.allclose(R @ R.T, np.eye(3), atol=1e-15)


def test_hcp_cuboid_of_reference_test():
    # the cuboid of test_lib_scene_generator_hcp_lattice_fill_cuboid: 8 x 8 x 8, r = 0.5
    c = S.hcp_fill_cuboid(8.0, 8.0, 8.0, 0.5)
    assert c.shape == (8 * 9 * 9, 3)
    # the (i, j, k) loop order and the centring offset -lattice(max)/2
    off = -S.hcp_lattice(7, 8, 8, 0.5) / 2
    assert np.allclose(c[0], off) and np.allclose(c[1], S.hcp_lattice(0, 0, 1, 0.5) + off)
    d = np.sqrt(((c[:, None, :] - c[None, :, :]) ** 2).sum(-1)) + np.eye(len(c)) * 9
    assert abs(d.min() - 1.0) < 1e-12                       # touching spheres, no overlap
    inner = np.all(np.abs(c - c.mean(0)) < 2.0, axis=1)
    assert np.all(np.sum(np.abs(d[inner] - 1.0) < 1e-9, axis=1) == 12)   # hcp: 12 neighbours


@pytest.mark.parametrize("R", [0.020, 0.035, 0.064])
def test_hcp_sphere_mask(R):
    r = 0.0076
    cub, inside = S.hcp_fill_sphere(R, r, (0, 0, 0), (0, 0, 1))
    rho = np.sqrt((cub ** 2).sum(1))
    assert np.array_equal(inside, (rho < R - r / 2) & (cub[:, 2] < 0))
    sc = S.hcp_sphere_scene(R)
    assert sc.n_spheres == int(inside.sum()) and sc.n_range == (1, 5)
    assert np.array_equal(sc.centres, cub[inside])


def test_plane_wave_field():
    pts = np.random.default_rng(1).uniform(-2, 2, (50, 3))
    jones = (math.cos(0.4), math.sin(0.4))
    E, H = fields.plane_wave_field(pts, 0.55, 1.0, 0.0, 0.0, jones)
    k = 2 * math.pi / 0.55
    assert np.allclose(E[:, 0], jones[0] * np.exp(-1j * k * pts[:, 2]), atol=1e-13)
    assert np.allclose(E[:, 2], 0)
    assert np.allclose(H * fields.Z_0, np.stack([-E[:, 1], E[:, 0], 0 * E[:, 0]], 1), atol=1e-13)
    # an oblique wave: E and H transverse to the propagation direction, |E| = 1
    th, ph = 0.7, 2.1
    E, H = fields.plane_wave_field(pts, 0.55, 1.33, th, ph, jones)
    assert np.allclose(np.sqrt((np.abs(E) ** 2).sum(1)), 1.0, atol=1e-13)
    kd = np.array([math.sin(th) * math.cos(ph), math.sin(th) * math.sin(ph), math.cos(th)])
    back = fields.rot_matrix(-math.pi / 2 - ph, -th, -math.pi / 2 - ph)
    kz = back @ np.array([0, 0, 1.0])          # the wave frame's z axis in world coordinates
    assert np.allclose(E @ kz, 0, atol=1e-13) and np.allclose(H @ kz, 0, atol=1e-13)
    assert kd.shape == (3,)


def _read_ppm(path):
    with open(path) as f:
        lines = [l for l in f.read().splitlines()]
    assert lines[0] == "P3"
    w, h = map(int, lines[1].split())
    body = [l for l in lines[3:] if not l.startswith("#")]
    vals = np.array(" ".join(body).split(), int)
    return w, h, vals.reshape(h, w, 3)


def test_ppm_and_csv_export(tmp_path):
    img = np.array([[1.0, -2.0, 0.0], [0.5, 4.0, -4.0]])   # 2 x 3: width 2, height 3
    p = str(tmp_path / "a.ppm")
    fields.write_ppm_p3(p, img)
    w, h, rgb = _read_ppm(p)
    assert (w, h) == (2, 3)
    # pixel (i, ii) is row ii, column i; +4 -> (255, 0, 0), -4 -> (0, 0, 255), 0 -> white
    assert tuple(rgb[1, 1]) == (255, 0, 0) and tuple(rgb[2, 1]) == (0, 0, 255)
    assert tuple(rgb[2, 0]) == (255, 255, 255)
    assert tuple(rgb[0, 0]) == (255, 255 - int(1 * 255.0 / 4), 255 - int(1 * 255.0 / 4))
    fields.write_ppm_p3(p, img, logarithmic=True)
    _, _, rgb = _read_ppm(p)
    lev = int(math.log(2.0 + 1) * 255.0 / math.log(5.0))
    assert tuple(rgb[1, 0]) == (255 - lev, 255 - lev, 255)
    c = str(tmp_path / "a.csv")
    fields.write_csv_array(c, img, ["u", "v", "w"])
    back = np.genfromtxt(c, delimiter=",", skip_header=1)
    assert np.array_equal(back, img)
    E = np.random.default_rng(0).standard_normal((4, 5, 3)) + 0j
    fields.field_export(E, E, str(tmp_path / "f"))
    names = sorted(os.listdir(tmp_path / "f"))
    assert len(names) == 30 and "poynting_abs_log.ppm" in names and "e_field_z.csv" in names


def test_plot_grid_matches_reference_counts():
    pts, nx, nz = hcp_benchmark.plot_grid(0.064)
    assert (nx, nz) == (200, 233)   # floor(3R / (3R/200)), floor(3.5R / (3R/200))
    assert pts.shape == (nx, nz, 3) and np.all(pts[..., 1] == 0)
