"""Timing of the reference's own runnable CPU code for this path: the legacy
SciPy solver, src/legacy/minimal_solver.py (ScalarDomain.calc_dndr :214-243,
dndr :245-259, solve :313-335, ray_at_exit :338-395), on the sinusoidal-slab
workload (128^3 over a 5 mm cube, ne = 1e24 m^-3 (1 + 0.1 sin(2 pi x / 0.5 mm)),
532 nm, 1e4 collimated rays with Gaussian positions of 1 mm 1/e^2 waist
entering at z = -2.5 mm).

Measurement infrastructure, not product code: it imports the reference from
/root/reference (present in the build container only) and prints one JSON
line. The solver runs unmodified through its own methods; two things are set
as its own init_beam would set them (the beam s0 and `extent`), and dndr is
wrapped to count right-hand-side evaluations.

What the numbers mean: solve() integrates all rays as one solve_ivp RK45
system with SciPy's default tolerances (rtol 1e-3, atol 1e-6), so every ray
takes the same few adaptive steps, and its time range
sqrt(x_max^2 + y_max^2 * z_max^2) / c covers about half the box (the
reference's expression). Rays/s is therefore the figure to quote; it is not
comparable step for step with a fixed-step tracer.

    python oracle/legacy_solver_timing.py [--rays 10000] [--reps 3]
"""
import argparse
import contextlib
import io
import json
import os
import sys
import time

os.environ.setdefault("OMP_NUM_THREADS", "1")
os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
os.environ.setdefault("MKL_NUM_THREADS", "1")

import numpy as np  # noqa: E402

REF_SRC = "/root/reference/src"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rays", type=int, default=10000)
    ap.add_argument("--reps", type=int, default=3)
    args = ap.parse_args()
    sys.path.insert(0, REF_SRC)
    import warnings
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", SyntaxWarning)
        from legacy import minimal_solver as ms

    n, ext = 128, 2.5e-3
    x = np.linspace(-ext, ext, n)
    dom = ms.ScalarDomain(x, x, x)
    XX = np.meshgrid(x, x, x, indexing="ij")[0]
    dom.external_ne(1e24 * (1.0 + 0.1 * np.sin(2 * np.pi * XX / 0.5e-3)))
    t0 = time.perf_counter()
    dom.calc_dndr(lwl=532e-9)
    t_setup = time.perf_counter() - t0
    dom.extent = ext                     # what init_beam sets for probing along z
    calls = [0]
    dndr = dom.dndr

    def counted(p):
        calls[0] += 1
        return dndr(p)
    dom.dndr = counted

    rng = np.random.default_rng(2024)
    N = args.rays
    s0 = np.zeros((6, N))
    s0[0:2] = rng.standard_normal((2, N)) * 0.5e-3
    s0[2] = -ext
    s0[5] = ms.c
    times = []
    for _ in range(args.reps):
        dom.s0 = s0.copy()
        calls[0] = 0
        t0 = time.perf_counter()
        with contextlib.redirect_stdout(io.StringIO()):   # the solver prints every ray's exit values
            dom.solve()
        times.append(time.perf_counter() - t0)
    t = float(np.median(times))
    print(json.dumps({
        "code": "src/legacy/minimal_solver.py ScalarDomain.solve (solve_ivp RK45, default tolerances)",
        "workload": f"128^3 sinusoidal slab, 532 nm, {N} rays, 5 mm cube",
        "rays": N, "seconds_median": t, "rays_per_s": N / t, "reps": args.reps,
        "rhs_evaluations": calls[0], "calc_dndr_seconds": t_setup,
        "mean_final_z_m": float(dom.sf[2].mean()),
        "threads": 1, "cpu_count": os.cpu_count()}))


if __name__ == "__main__":
    main()
