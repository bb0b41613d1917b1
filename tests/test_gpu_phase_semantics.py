"""The phase of the FP64 tracer has the legacy solver's semantics.

The legacy full solver integrates omega * (n - 1) with n interpolated from
the refractive index on the grid points (src/legacy/full_solver.py:289,
:342-345). The trace layout of the packed grid carries n - 1 at the grid
points and the tracers interpolate it, so they follow those semantics. The
oracle's reference form (phase_mode='reference') is pinned to the legacy
solver's own ScalarDomain.phase by tests/golden/phase.npz
(test_oracle_golden.py); here the FP64 kernel's accumulated phase is held to
it along the same trajectories, at the 128^3 sinusoidal slab (whole-
configuration rays) and the 512^3 Kolmogorov box (a ray subset the numpy
oracle follows in seconds). The other form, n from the interpolated density,
differs from it at O(h^2); that gap is stated too: 3.4e-8 (slab) and 4.8e-7
(Kolmogorov box) of the largest phase, measured with the oracle.
"""
import math

import numpy as np
import pytest

from helpers import C, run_kernel
from oracle import ref_restated as rr
from sloth_b200 import runtime, workloads

pytestmark = pytest.mark.gpu

L = 5e-3
OMEGA = 2 * np.pi * C / 532e-9


def _phases(ne, rays, n):
    h = L / (n - 1)
    sched = runtime.schedule_times(np.array([math.sqrt(8.0) * L]), (h, h, h))
    kw = dict(project=True, plane=L / 2)
    k = run_kernel(ne.astype(np.float32), rays.astype(np.float32), (-L / 2,) * 3, (h,) * 3, OMEGA, sched,
                   precision="f64", want_state=False, **kw)
    grid = rr.Grid(ne.astype(np.float32).astype(np.float64), (-L / 2,) * 3, (h,) * 3, OMEGA)
    okw = dict(dtau=sched.dtau, first_save=sched.first_save, save_every=sched.save_every, n_saves=sched.n_saves,
               **kw)
    r64 = rays.astype(np.float32).astype(np.float64)
    ref = rr.trace_rays(grid, r64, phase_mode="reference", **okw)["phase"][-1]
    dens = rr.trace_rays(grid, r64, phase_mode="density", **okw)["phase"][-1]
    scale = np.abs(ref).max()
    return np.abs(k["phase"][-1] - ref).max() / scale, np.abs(dens - ref).max() / scale


def test_phase_semantics_sinusoid_slab_128():
    n = 128
    ne = workloads.sinusoid_slab(n, L=L, n0=1e24).double().numpy()
    rays = workloads.gaussian_beam(10_000, waist=1e-3, L=L, seed=101).numpy()[:, ::5]
    kernel_err, density_gap = _phases(ne, rays, n)
    assert kernel_err < 1e-10                 # the kernel follows the legacy semantics
    assert density_gap < 1e-7                 # the other semantics, measured 3.4e-8


def test_phase_semantics_kolmogorov_512():
    n = 512
    ne = workloads.kolmogorov_box(n, L=L, mean=1e25, rms=0.2, seed=2024, device="cuda").cpu().double().numpy()
    rays = workloads.gaussian_beam(10_000, waist=1.5e-3, L=L, seed=2025).numpy()[:, :100]
    kernel_err, density_gap = _phases(ne, rays, n)
    assert kernel_err < 1e-10
    assert density_gap < 1e-6                 # measured 4.8e-7
