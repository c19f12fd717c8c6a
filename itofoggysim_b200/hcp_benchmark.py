"""The reference's own benchmark: hcp-packed half-sphere clusters of growing radius, solved with the
ML-FMM and with the direct (T-matrix) operator, and the scattered and total field plotted on an
x-z plane (lib_mie_ms_benchmark, FoggySim/src/lib/mie_theory/lib_mie_multi_sphere.f90:3717-4164).

    python -m itofoggysim_b200.hcp_benchmark --out hcp_out [--steps 12] [--operator both]
        [--no-plot] [--first-step 1]

For step i = 1..steps the cluster radius is 20 nm + (i - 1) (64 - 20) nm / steps, filled with
7.5 nm particles (n = 2.5287) on a 7.6 nm hcp lattice (itofoggysim_b200.scene.hcp_sphere_scene).
Each step solves with the single-sphere initial guess (GMRES(10) to 1e-6, the reference defaults),
timing CPU and wall clock around the solve, then evaluates the scattered field on the grid
x in [-1.5 R, 1.5 R), z in [-1.5 R, 2 R), y = 0, step 3 R / 200 (foggy_get_field, on the GPU),
exports it with lib_field_export's file set (scattered in <out>/<operator>/step_<i>/real/, plus the
incident plane wave in .../realTotal/), and times that too.  Per operator it writes the
reference's table hcp_sphere_benchmark_ml_fmm.csv / hcp_sphere_benchmark_t_matrix.csv with the
columns no_spheres, calc: CPU-Time, calc: WALL-Time, plot: CPU-Time, plot: WALL-Time, and the
sphere centres of the last step in hcp_sphere.csv.

The reference's plot loop calls lib_mie_ms_get_field once per point and adds the incident wave
evaluated at the point itself (not shifted by the wave's origin d_0_i, which its right-hand side
does use); both are kept as the reference has them.
"""
import argparse
import os
import time

import numpy as np


def plot_grid(sphere_radius):
    """Sample points of the reference's field plot (x-major, then z)."""
    x0, x1 = -sphere_radius * 1.5, sphere_radius * 1.5
    z0, z1 = -sphere_radius * 1.5, sphere_radius * 2.0
    step = (x1 - x0) / 200.0
    nx = abs(int(np.floor((x1 - x0) / step)))
    nz = abs(int(np.floor((z1 - z0) / step)))
    xs = x0 + np.arange(nx) * step
    zs = z0 + np.arange(nz) * step
    X, Z = np.meshgrid(xs, zs, indexing="ij")
    pts = np.stack([X, np.zeros_like(X), Z], axis=-1)
    return pts, nx, nz


def run_step(sphere_radius, use_ml_fmm, plot, out_dir, tree_l_max=0):
    from . import fields, scene as S, solver
    sc = S.hcp_sphere_scene(sphere_radius)
    sc.tree_l_max = tree_l_max
    res = np.zeros(5)
    res[0] = sc.n_spheres
    c0, w0 = time.process_time(), time.perf_counter()
    with solver.MultiSphereSolver(sc, use_ml_fmm=use_ml_fmm, init_with_single_sphere=True) as s:
        x, st = s.solve(raise_on_error=False)
        res[1] = time.process_time() - c0
        res[2] = time.perf_counter() - w0
        if plot:
            c1, w1 = time.process_time(), time.perf_counter()
            pts, nx, nz = plot_grid(sphere_radius)
            E, H = s.get_field(x, pts.reshape(-1, 3))
            E = E.reshape(nx, nz, 3)
            H = H.reshape(nx, nz, 3)
            fields.field_export(E, H, os.path.join(out_dir, "real"))
            jones = (complex(sc.jones[0, 0], sc.jones[0, 1]), complex(sc.jones[0, 2], sc.jones[0, 3]))
            Ei, Hi = fields.plane_wave_field(pts.reshape(-1, 3), sc.lambda_0, sc.n_medium,
                                             float(sc.wave_theta[0]), float(sc.wave_phi[0]), jones)
            fields.field_export(E + Ei.reshape(nx, nz, 3), H + Hi.reshape(nx, nz, 3),
                                os.path.join(out_dir, "realTotal"))
            res[3] = time.process_time() - c1
            res[4] = time.perf_counter() - w1
    return res, sc, st


HEADER = ["no_spheres", "calc: CPU-Time", "calc: WALL-Time", "plot: CPU-Time", "plot: WALL-Time"]


def main(argv=None):
    from . import fields
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default="hcp_out")
    ap.add_argument("--steps", type=int, default=12)
    ap.add_argument("--first-step", type=int, default=1)
    ap.add_argument("--last-step", type=int, default=0)
    ap.add_argument("--operator", choices=["mlfmm", "direct", "both"], default="both")
    ap.add_argument("--no-plot", action="store_true")
    args = ap.parse_args(argv)
    r0, r1 = 0.020, 0.064
    step = (r1 - r0) / args.steps
    last = args.last_step or args.steps
    ops = [("ml_fmm", True), ("t_matrix", False)]
    if args.operator != "both":
        ops = [o for o in ops if o[1] == (args.operator == "mlfmm")]
    os.makedirs(args.out, exist_ok=True)
    for name, fmm in ops:
        table = np.zeros((args.steps, 5))
        for i in range(args.first_step, last + 1):
            R = r0 + step * (i - 1)
            res, sc, st = run_step(R, fmm, not args.no_plot, os.path.join(args.out, name, "step_%d" % i))
            table[i - 1] = res
            print("%s step %d: R = %.1f nm, %d spheres, n_max %d, %d iterations, backward error %.2e, "
                  "calc %.3f s, plot %.3f s" % (name, i, R * 1e3, sc.n_spheres, sc.n_range[1],
                                                st["iterations"], st["backward_error"], res[2], res[4]),
                  flush=True)
            fields.write_csv_array(os.path.join(args.out, "hcp_sphere_benchmark_%s.csv" % name), table, HEADER)
            fields.write_csv_array(os.path.join(args.out, "hcp_sphere.csv"), sc.centres)


if __name__ == "__main__":
    main()
