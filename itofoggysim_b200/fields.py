"""Field helpers around foggy_get_field: the incident plane-wave field, and the reference's field
export to PPM images and CSV tables.

  rot_matrix            lib_math_get_matrix_rot      libmath/src/math/lib_math_type_operator.f90:1768-1810
  plane_wave_field      lib_field_plane_wave_get_field / _scalar
                                                    FoggySim/src/lib/field/lib_field_plane_wave.f90
  field_export          lib_field_export             FoggySim/src/lib/field/lib_field.f90:35-260
  write_ppm_p3          write_ppm_p3, color_map_temperature
                                                    libtoolbox/src/file_io.f90:131-247
  write_csv_array       write_csv_real_array         libtoolbox/src/file_io.f90:314-358

These run on the host: they format or add closed-form values to what the device returns.
"""
import math
import os

import numpy as np

Z_0 = 376.730313668     # free-space wave impedance [Ohm] (lib_constants.f90)


def rot_matrix(phi, theta, psi):
    """Euler rotation in the x-convention (the reference's lib_math_get_matrix_rot)."""
    cph, sph = math.cos(phi), math.sin(phi)
    cth, sth = math.cos(theta), math.sin(theta)
    cps, sps = math.cos(psi), math.sin(psi)
    return np.array([[cps * cph - cth * sph * sps, cps * sph + cth * cph * sps, sps * sth],
                     [-sps * cph - cth * sph * cps, -sps * sph + cth * cph * cps, cps * sth],
                     [sth * sph, -sth * cph, cth]])


def plane_wave_field(points, lambda_0, n_medium=1.0, theta=0.0, phi=0.0, jones=(1.0, 0.0),
                     e_field_0=1.0, phase=0.0, convention=1):
    """E and H (complex, (npoints, 3)) of a plane wave at points, as lib_field_plane_wave_get_field
    evaluates it: rotate the point into the wave frame, E = e0 exp(-+i(k z - phase)) (Jones x, y, 0),
    H = R(-pi/2, 0, 0) E n / Z_0, rotated back."""
    pts = np.asarray(points, np.float64).reshape(-1, 3)
    rotate = phi != 0.0 or theta != 0.0
    if rotate:
        pts = pts @ rot_matrix(math.pi / 2.0 + phi, theta, math.pi / 2.0 + phi).T
    arg = -2.0 * math.pi * pts[:, 2] * n_medium / lambda_0 + phase
    f = e_field_0 * np.exp(1j * arg) if convention == 1 else e_field_0 * np.exp(-1j * arg)
    E = np.zeros((len(pts), 3), np.complex128)
    E[:, 0] = f * complex(jones[0])
    E[:, 1] = f * complex(jones[1])
    H = (E @ rot_matrix(-math.pi / 2.0, 0.0, 0.0).T) / (Z_0 / n_medium)
    if rotate:
        back = rot_matrix(-math.pi / 2.0 - phi, -theta, -math.pi / 2.0 - phi)
        E = E @ back.T
        H = H @ back.T
    return E, H


def _fortran_int(v, w):
    return ("%d" % v).rjust(w)


def _eng(v):
    """Engineering notation with two decimals (the reference's EN17.2 header field)."""
    if v == 0 or not math.isfinite(v):
        return ("%.2f" % v).rjust(17)
    e = int(math.floor(math.log10(abs(v)) / 3.0)) * 3
    m = v / 10.0 ** e
    if abs(m) >= 999.995:
        e += 3
        m = v / 10.0 ** e
    return ("%.2fE%+03d" % (m, e)).rjust(17)


def color_map_temperature(img, max_value=255, logarithmic=False):
    """RGB of each pixel: positive values fade white -> red, negative white -> blue, zero white,
    scaled by the largest magnitude (optionally log(1 + |v|))."""
    img = np.asarray(img, np.float64)
    top = max(abs(img.max()), abs(img.min()))
    rgb = np.full(img.shape + (3,), max_value, np.int64)
    a = np.abs(img)
    if logarithmic:
        with np.errstate(divide="ignore", invalid="ignore"):
            lev = np.log(a + 1.0) * float(np.float32(max_value)) / math.log(top + 1.0)
    else:
        with np.errstate(divide="ignore", invalid="ignore"):
            lev = a * float(np.float32(max_value)) / top
    lev = np.where(np.isfinite(lev), lev, 0.0).astype(np.int64)   # Fortran int() truncates
    pos, neg = img > 0, img < 0
    rgb[pos, 1] = max_value - lev[pos]
    rgb[pos, 2] = max_value - lev[pos]
    rgb[neg, 0] = max_value - lev[neg]
    rgb[neg, 1] = max_value - lev[neg]
    return rgb


def write_ppm_p3(path, img, logarithmic=False):
    """ASCII RGB image of a 2-D array: width = first index, one image row per second index, ten
    RGB triplets per text line, as write_ppm_p3 writes it."""
    img = np.asarray(img, np.float64)
    rgb = color_map_temperature(img, 255, logarithmic)
    with open(path, "w") as f:
        f.write("P3\n")
        f.write(_fortran_int(img.shape[0], 6) + " " + _fortran_int(img.shape[1], 6) + "\n")
        f.write("255\n")
        f.write("# The part above is the header\n")
        f.write("# P3   means this is a RGB color image in ASCII\n")
        f.write("# " + _fortran_int(img.shape[0], 6) + " x " + _fortran_int(img.shape[1], 6)
                + "  is the width and height of the image in pixels\n")
        f.write("# pixel value range for each color: 0 - 255\n")
        f.write("# data point value range: " + _eng(img.min()) + " - " + _eng(img.max()) + "\n")
        f.write("# The part below is image data: RGB triplets\n")
        for ii in range(img.shape[1]):
            vals = rgb[:, ii, :].reshape(-1)
            for s in range(0, len(vals), 30):
                f.write("".join("%3d " % v for v in vals[s:s + 30]) + "\n")


def write_csv_array(path, c, header=None):
    """One text line per first index, ES25.16 values separated by commas."""
    c = np.asarray(c, np.float64)
    with open(path, "w") as f:
        if header:
            f.write(" " + ",".join(h.strip() for h in header) + "\n")
        for row in c:
            f.write(",".join("%25.16E" % v for v in row) + " \n")


def poynting(E, H):
    """Time-averaged Poynting vector Re(E x H*) / 2 and its length."""
    S = np.real(np.cross(E, np.conj(H))) / 2.0
    return S, np.sqrt(np.sum(S * S, axis=-1))


def field_export(E, H, path):
    """The files lib_field_export writes for fields sampled on a 2-D grid (arrays (nx, nz, 3)):
    real parts of E and H per component and the Poynting vector, as PPM images (linear and
    logarithmic) and CSV tables."""
    os.makedirs(path, exist_ok=True)
    E = np.asarray(E)
    H = np.asarray(H)
    S, S_abs = poynting(E, H)
    planes = {}
    for c, name in enumerate("xyz"):
        planes["e_field_" + name] = np.real(E[..., c])
        planes["h_field_" + name] = np.real(H[..., c])
        planes["poynting_" + name] = S[..., c]
    for key in ["e_field_x", "e_field_y", "e_field_z", "h_field_x", "h_field_y", "h_field_z",
                "poynting_x", "poynting_y", "poynting_z"]:
        write_ppm_p3(os.path.join(path, key + ".ppm"), planes[key])
        write_ppm_p3(os.path.join(path, key + "_log.ppm"), planes[key], logarithmic=True)
    write_ppm_p3(os.path.join(path, "poynting_abs.ppm"), S_abs)
    write_ppm_p3(os.path.join(path, "poynting_abs_log.ppm"), S_abs, logarithmic=True)
    for key in ["e_field_x", "e_field_y", "e_field_z", "h_field_x", "h_field_y", "h_field_z",
                "poynting_x", "poynting_y", "poynting_z"]:
        write_csv_array(os.path.join(path, key + ".csv"), planes[key])
    write_csv_array(os.path.join(path, "poynting_abs.csv"), S_abs)
    return True
