"""The phase of the FP64 tracer against the legacy solver's phase semantics.

The legacy full solver integrates omega * (n - 1) with n interpolated from
the refractive index on the grid points (src/legacy/full_solver.py:289,
:342-345); the tracers take n from the interpolated density. The oracle has
both forms (`phase_mode`), and its reference form is pinned to the legacy
solver's own ScalarDomain.phase by tests/golden/phase.npz
(test_oracle_golden.py). Here the FP64 kernel's accumulated phase is compared
with the oracle's reference-form phase along the same trajectories, at the
128^3 sinusoidal slab (whole-configuration rays) and the 512^3 Kolmogorov box
(a ray subset the numpy oracle follows in seconds). The difference is the
O(h^2) gap between the two semantics; measured: 3.4e-8 (slab) and 4.8e-7
(Kolmogorov box) of the largest phase.
"""
import math

import numpy as np
import pytest
import torch

from helpers import C, run_kernel
from oracle import ref_restated as rr
from sloth_b200 import runtime, workloads

pytestmark = pytest.mark.gpu

L = 5e-3
OMEGA = 2 * np.pi * C / 532e-9


def _gap(ne, rays, n):
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
    same = rr.trace_rays(grid, r64, phase_mode="kernel", **okw)["phase"][-1]
    scale = np.abs(ref).max()
    return (np.abs(k["phase"][-1] - ref).max() / scale, np.abs(k["phase"][-1] - same).max() / scale)


def test_phase_semantics_gap_sinusoid_slab_128():
    n = 128
    ne = workloads.sinusoid_slab(n, L=L, n0=1e24).double().numpy()
    rays = workloads.gaussian_beam(10_000, waist=1e-3, L=L, seed=101).numpy()[:, ::5]
    gap, same = _gap(ne, rays, n)
    assert same < 1e-10                       # the kernel follows its own semantics exactly
    assert gap < 1e-7                         # measured 3.4e-8


def test_phase_semantics_gap_kolmogorov_512():
    n = 512
    ne = workloads.kolmogorov_box(n, L=L, mean=1e25, rms=0.2, seed=2024, device="cuda").cpu().double().numpy()
    rays = workloads.gaussian_beam(10_000, waist=1.5e-3, L=L, seed=2025).numpy()[:, :100]
    gap, same = _gap(ne, rays, n)
    assert same < 1e-10
    assert gap < 1e-6                         # measured 4.8e-7
