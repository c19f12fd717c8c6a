"""Operator applications on a lognormal sphere cluster, for timing and profiling runs.

    python -m itofoggysim_b200.operator_case --spheres 400 --applications 1

builds the lognormal water-sphere scene (median radius 0.6 um, sigma_ln 0.3, lambda 0.55 um,
per-sphere Wiscombe orders) with the given number of spheres in a cube whose edge keeps the
2000-sphere / 40 um volume fraction, and applies the direct operator y = A x to the right-hand
side on cuda:0.  The first application also builds the pair tables.  Each application prints
its wall time.

    python -m itofoggysim_b200.operator_case --spheres 300 --solve [--precision mixed]

solves the same scene instead (GMRES(50) to 1e-8, FP64 or mixed precision) and prints the wall
time, iterations and backward error; in mixed precision the Arnoldi steps launch the FP32
operator, the run used to profile it.
"""
import argparse
import time

import numpy as np


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--spheres", type=int, default=400)
    ap.add_argument("--applications", type=int, default=1)
    ap.add_argument("--pair-tables", type=int, default=0, help="0 auto, -1 off")
    ap.add_argument("--solve", action="store_true", help="one GMRES solve instead of applications")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    args = ap.parse_args(argv)

    import torch
    from . import scene as S, solver

    n = args.spheres
    sc = S.medium_cluster(n=n, box=40.0 * (n / 2000.0) ** (1.0 / 3.0))
    s = solver.MultiSphereSolver(sc, pair_tables=args.pair_tables,
                                 precision=1 if args.precision == "mixed" else 0)
    if args.solve:
        s.set_restart(50)
        s.set_tolerance(1e-8)
        t0 = time.perf_counter()
        _, st = s.solve()
        print("solve (%s): %.2f ms, %d iterations, backward error %.2e"
              % (args.precision, (time.perf_counter() - t0) * 1e3, st["iterations"], st["backward_error"]),
              flush=True)
        s.close()
        return
    x = torch.zeros(2 * s.n, dtype=torch.float64, device="cuda:0")
    y = torch.zeros_like(x)
    x.copy_(torch.from_numpy(s.get_vector_b().view(np.float64)))
    for i in range(args.applications):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s.matvec_device(x.data_ptr(), y.data_ptr())
        torch.cuda.synchronize()
        print("application %d: %.2f ms" % (i, (time.perf_counter() - t0) * 1e3), flush=True)
    s.close()


if __name__ == "__main__":
    main()
