"""The oracle's exit step: a step cut at a face samples its stage points
clamped into the grid, so all four stages see the field's limit from inside.

On a 128^3 grid the 4th stage of the exit step lands on the far face up to
rounding. A clamp done in metres maps back to a cell coordinate just above
n - 1 there, and would sample the fill value 0 for that stage. The test
checks, for the C and the numpy oracle, that the exit step's change of the
transverse velocity is the cut fraction phi times a full step's, as it is
when every stage samples the field, and not (1 - 1/6) of that."""
import numpy as np
import pytest

from oracle import oracle_c
from oracle import ref_restated as rr
from sloth_b200 import runtime, workloads
from sloth_b200.core import physics

L = 5e-3
OMEGA = 2 * np.pi * physics.C / 532e-9


@pytest.mark.parametrize("which", ["c", "numpy"])
def test_exit_step_samples_every_stage_inside(which):
    n = 128
    h = L / (n - 1)
    ne = workloads.sinusoid_slab(n, L=L, n0=1e24).numpy().astype(np.float64)
    rays = workloads.gaussian_beam(4, waist=1e-3, L=L, seed=101).numpy().astype(np.float64)
    base = runtime.schedule_times(np.array([np.sqrt(8.0) * L]), (h, h, h))
    grid = rr.Grid(ne, (-L / 2,) * 3, (h,) * 3, OMEGA)
    kw = dict(dtau=base.dtau, first_save=250, save_every=1, n_saves=8)
    out = oracle_c.trace_rays(grid, rays, **kw) if which == "c" else rr.trace_rays(grid, rays, **kw)
    z = (out["state"][:, 2] + L / 2) / h            # cells along the probing axis, (saves, rays)
    vx = out["state"][:, 3]
    for r in range(rays.shape[1]):
        j = int(np.argmax(z[:, r] > n - 1))          # first save after the exit
        assert 1 <= j < 7
        w = z[j - 1, r] - z[j - 2, r]               # cells per full step
        phi = (n - 1 - z[j - 1, r]) / w
        full = vx[j - 1, r] - vx[j - 2, r]          # the last full step's change
        cut = vx[j, r] - vx[j - 1, r]
        assert 0.0 < phi < 1.0
        assert abs(cut / full - phi) < 0.02 * phi, (cut / full, phi)
