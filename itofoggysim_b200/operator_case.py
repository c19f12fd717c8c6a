"""Operator applications on a lognormal sphere cluster, for timing and profiling runs.

    python -m itofoggysim_b200.operator_case --spheres 400 --applications 1

builds the lognormal water-sphere scene (median radius 0.6 um, sigma_ln 0.3, lambda 0.55 um,
per-sphere Wiscombe orders) with the given number of spheres in a cube whose edge keeps the
2000-sphere / 40 um volume fraction, and applies the direct operator y = A x to the right-hand
side on cuda:0.  The first application also builds the pair tables.  Each application prints
its wall time.
"""
import argparse
import time

import numpy as np


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--spheres", type=int, default=400)
    ap.add_argument("--applications", type=int, default=1)
    ap.add_argument("--pair-tables", type=int, default=0, help="0 auto, -1 off")
    args = ap.parse_args(argv)

    import torch
    from . import scene as S, solver

    n = args.spheres
    sc = S.medium_cluster(n=n, box=40.0 * (n / 2000.0) ** (1.0 / 3.0))
    s = solver.MultiSphereSolver(sc, pair_tables=args.pair_tables)
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
