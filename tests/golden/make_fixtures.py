"""Generate the golden fixtures in this folder from the reference's own test data.

Run once, in a checkout where the reference project is available:

    python tests/golden/make_fixtures.py /path/to/reference

It copies the Mathematica-generated translation-coefficient tables and extracts the inline
golden values of the reference's Fortran unit tests (read as text, never compiled):

  * ground_truth_AB_mnmunu.csv, ground_truth_AB_mnmunu_minus_phi.csv
      FoggySim/ground_truth/lib_math_vector_spherical_harmonics/ (x=2, theta=0.5, phi=0.5 and
      phi=2*pi-0.5, n,nu <= 5, z=3; consumed at
      libmath/src/math/lib_math_vector_spherical_harmonics.f90:2876-3168)
  * ground_truth_M_mn.csv, ground_truth_N_mn.csv
      same folder (theta=0.2, phi=0, k=2 pi, r=50, z=3, n <= 4; consumed at
      libmath/src/math/lib_math_vector_spherical_harmonics.f90:2443-2575, tolerance 1e-13)
  * inline_goldens.json with
      wigner_3j          libmath/src/math/lib_math_wigner.f90:140-164
      ab_xu_cruzan       libmath/src/math/lib_math_vector_spherical_harmonics.f90:2799-2875
      sph_jn_x5          libmath/src/math/lib_math_bessel.f90:2433-2517
      riccati_xi_x05     libmath/src/math/lib_math_bessel.f90:3536-3633
      pi_tau_theta2      libmath/src/math/lib_math_legendre.f90:2099-2210
      mie_ab_m15_x10     FoggySim/src/lib/mie_theory/lib_mie_ss_helper_functions.f90:1639-1703
      universal_index    libtree/src/lib/lib_tree_helper_functions.f90:2166-2204
      tree_neighbours    libtree/src/lib/lib_tree_helper_functions.f90:2438-2470, 2529-2560
      tree_parent        libtree/src/lib/lib_tree_helper_functions.f90:2277-2310
      tree_children      libtree/src/lib/lib_tree_helper_functions.f90:2312-2356

The tests read only the files written here, so they run where the reference is absent.
"""
import json
import os
import re
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def fnum(tok):
    tok = tok.strip().replace("_8", "").replace("D", "e").replace("d", "e")
    return float(tok)


def lines(path, a, b):
    with open(path) as f:
        return f.read().splitlines()[a - 1:b]


def data_block(path, a, b, name):
    txt = "\n".join(lines(path, a, b))
    m = re.search(r"data\s+" + name + r"\s*/(.*?)/\s*$", txt, re.S | re.M)
    body = re.sub(r"&", " ", m.group(1))
    return body


def main(ref):
    vsh = os.path.join(ref, "FoggySim/ground_truth/lib_math_vector_spherical_harmonics")
    for fn in ("ground_truth_AB_mnmunu.csv", "ground_truth_AB_mnmunu_minus_phi.csv", "ground_truth_M_mn.csv",
               "ground_truth_N_mn.csv"):
        shutil.copyfile(os.path.join(vsh, fn), os.path.join(HERE, fn))

    g = {}
    # Wigner 3j (Mathematica values, tolerance 1e-14)
    wig = os.path.join(ref, "libmath/src/math/lib_math_wigner.f90")
    vals = [fnum(m.group(1)) for l in lines(wig, 160, 164)
            for m in [re.search(r"=\s*([-+0-9.eEdD_]+)", l)] if m]
    g["wigner_3j"] = {"j1": 98, "j2": 115, "j3": [213, 212, 211, 210, 209],
                      "m1": -69, "m2": -100, "m3": 169, "values": vals, "tol": 1e-14}

    # Xu / Cruzan a and b coefficients
    vshf = os.path.join(ref, "libmath/src/math/lib_math_vector_spherical_harmonics.f90")
    ga, gb = {}, {}
    for l in lines(vshf, 2825, 2845):
        m = re.search(r"ground_truth_([ab])\((\d)\)\s*=\s*([-+0-9.eEdD_]+)", l)
        if m:
            (ga if m.group(1) == "a" else gb)[int(m.group(2))] = fnum(m.group(3))
    g["ab_xu_cruzan"] = {"m": 15, "n": 16, "mu": -15, "nu": 20, "q": [1, 2, 3, 4, 5],
                         "a": [ga[i] for i in range(1, 6)], "b": [gb[i] for i in range(1, 6)],
                         "tol": 1e-13}

    # spherical Bessel j_n(5), n = 0..40 (relative tolerance 1e-13)
    bes = os.path.join(ref, "libmath/src/math/lib_math_bessel.f90")
    body = data_block(bes, 2455, 2500, "ground_truth_j")
    g["sph_jn_x5"] = {"x": 5.0, "values": [fnum(t) for t in body.split(",")], "tol": 1e-13}

    # Riccati xi_n(0.5) = 0.5 h_n^(1)(0.5), n = 0..40
    body = data_block(bes, 3565, 3615, "ground_truth_xi")
    pairs = re.findall(r"\(([^,]+),([^)]+)\)", body)
    g["riccati_xi_x05"] = {"x": 0.5, "re": [fnum(a) for a, _ in pairs],
                           "im": [fnum(b) for _, b in pairs], "tol": 1e-13}

    # pi_nm / tau_nm at theta = 2 with Condon-Shortley phase
    leg = os.path.join(ref, "libmath/src/math/lib_math_legendre.f90")
    pi, tau = {}, {}
    for l in lines(leg, 2120, 2175):
        m = re.search(r"ground_truth_(pi|tau)_nm%item\((\d)\)%item\(\s*(-?\d)\)\s*=\s*([-+0-9.eEdD_]+)", l)
        if m:
            (pi if m.group(1) == "pi" else tau)["%s,%s" % (m.group(2), m.group(3))] = fnum(m.group(4))
    g["pi_tau_theta2"] = {"theta": 2.0, "n_max": 3, "cs_phase": True, "pi": pi, "tau": tau,
                          "tol_pi": 1e-13, "tol_tau": 5e-5}  # reference: 5e-5 absolute (lib_math_legendre.f90:1023)

    # Mie a_n, b_n for m = 1.5, x = 10 (Barber & Hill program S2, relative 1e-6)
    mie = os.path.join(ref, "FoggySim/src/lib/mie_theory/lib_mie_ss_helper_functions.f90")
    ab = {"a": {}, "b": {}}
    for l in lines(mie, 1660, 1680):
        m = re.search(r"ground_truth_([ab])_n\((\d)\)\s*=\s*cmplx\(([^,]+),([^,]+),", l)
        if m:
            ab[m.group(1)][int(m.group(2))] = [fnum(m.group(3)), fnum(m.group(4))]
    g["mie_ab_m15_x10"] = {"m": 1.5, "x": 10.0, "n": [1, 2, 3, 4],
                           "a": [ab["a"][i] for i in range(1, 5)],
                           "b": [ab["b"][i] for i in range(1, 5)], "tol": 1e-6}

    # universal index of (0.75, 0.5, 2^-9 + 2^-8) at level 1 is 6 (3-D build)
    g["universal_index"] = [{"point": [0.75, 0.5, 2.0 ** -9 + 2.0 ** -8], "l": 1, "n": 6}]

    # neighbours at distance 1 (3-D build): the ground-truth arrays, -1 marks an unused slot
    tre = os.path.join(ref, "libtree/src/lib/lib_tree_helper_functions.f90")

    def int_array(a, b):
        txt = "\n".join(lines(tre, a, b))
        m = re.search(r"neighbour_all_ground_truth\s*=\s*\(/(.*?)/\)", txt, re.S)
        return [int(t) for t in re.sub(r"&", " ", m.group(1)).replace("\n", " ").split(",")]

    g["tree_neighbours"] = [{"l": 2, "n": 35, "neighbours": [v for v in int_array(2438, 2472) if v >= 0]},
                            {"l": 1, "n": 5, "neighbours": [v for v in int_array(2529, 2562) if v >= 0]}]
    par = [int(m.group(1)) for l in lines(tre, 2290, 2296) for m in [re.search(r"n_parent_ground_trouth\s*=\s*(\d+)", l)] if m]
    g["tree_parent"] = {"l": 1, "n": 6, "parent": par[-1]}
    kids = [int(m.group(1)) for l in lines(tre, 2330, 2340) for m in [re.search(r"children_n_ground_truth\(\d\)\s*=\s*(\d+)", l)] if m]
    g["tree_children"] = {"n": 1, "children": kids[-8:]}

    with open(os.path.join(HERE, "inline_goldens.json"), "w") as f:
        json.dump(g, f, indent=1)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FOGGY_REFERENCE")
    if not ref:
        sys.exit("usage: make_fixtures.py REFERENCE_CHECKOUT (or set FOGGY_REFERENCE)")
    main(ref)
