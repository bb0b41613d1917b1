"""Shared builders for the parity tests: one seeded case, traced by the CUDA
kernels through the C ABI and by the oracle on the same inputs."""
from __future__ import annotations

import numpy as np
import torch

from oracle import oracle_c
from oracle import ref_restated as rr
from sloth_b200 import runtime, workloads
from sloth_b200.core import physics

C = physics.C


def case(kind, n, nrays, *, seed=0, lwl=532e-9, L=5e-3, axis=2, jitter=0.0, waist=2e-3):
    """(ne float32 numpy (n,n,n), rays float32 numpy (6,N), origin, spacing, omega)."""
    if kind == "sinusoid":
        ne = workloads.sinusoid_slab(n, L=L)
    elif kind == "trough":
        ne = workloads.parabolic_trough(n, L=L)
    elif kind == "kolmogorov":
        ne = workloads.kolmogorov_box(n, L=L, seed=seed)
    elif kind == "vacuum":
        ne = torch.zeros((n, n, n), dtype=torch.float32)
    else:
        raise ValueError(kind)
    rays = workloads.gaussian_beam(nrays, waist=waist, L=L, jitter=jitter, seed=seed + 1)
    if axis != 2:
        # relabel the axes so that the case probes along `axis`: old axis a
        # becomes new axis to_new[a], and new axis k holds old axis order[k]
        to_new = {0: {0: 1, 1: 2, 2: 0}, 1: {0: 0, 1: 2, 2: 1}}[axis]
        order = {0: (2, 0, 1), 1: (0, 2, 1)}[axis]
        ne = ne.permute(*order)
        r = rays.clone()
        for a in range(3):
            r[to_new[a]] = rays[a]
            r[3 + to_new[a]] = rays[3 + a]
        rays = r
    ne = ne.contiguous().numpy()
    h = L / (n - 1)
    return ne, rays.numpy(), (-L / 2,) * 3, (h,) * 3, 2 * np.pi * C / lwl


def oracle_grid(ne, origin, spacing, omega, Te=None, Z=None):
    return rr.Grid(ne.astype(np.float64), origin, spacing, omega, Te=Te, Z=Z)


def run_kernel(ne, rays, origin, spacing, omega, sched, *, precision, axis=2, project=False, plane=0.0,
               inv_brems=False, Te=None, Z=None, want_state=True, integrator="rkn"):
    g = runtime.pack_grid(torch.from_numpy(ne), origin, spacing, omega, precision=precision)
    dt = torch.float32 if precision == "f32" else torch.float64
    r = torch.from_numpy(rays).to("cuda", dt)
    out = runtime.trace(g, r, sched, axis=axis, project=project, plane=plane, inv_brems=inv_brems, Te=Te, Z=Z,
                        want_state=want_state, integrator=integrator)
    torch.cuda.synchronize()
    res = {k: v.cpu().numpy() for k, v in out.items()}
    res["total_steps"] = int(res["total_steps"][0])
    return res


def run_oracle(ne, rays, origin, spacing, omega, sched, *, axis=2, project=False, plane=0.0, inv_brems=False,
               Te=None, Z=None, integrator="rkn"):
    grid = oracle_grid(ne, origin, spacing, omega, Te=Te, Z=Z)
    return oracle_c.trace_rays(grid, rays.astype(np.float64), dtau=sched.dtau, first_save=sched.first_save,
                               save_every=sched.save_every, n_saves=sched.n_saves, axis=axis, project=project,
                               plane=plane, inv_brems=inv_brems, integrator=integrator)


def position_error(got_state, ref_state, L):
    """max over rays and saves of |dx| / L (positions rows 0..2)."""
    d = np.abs(np.asarray(got_state, np.float64)[:, :3] - ref_state[:, :3])
    return d.max() / L


def direction_error(got_state, ref_state):
    """max |d(v/c)| over rays and saves."""
    d = np.abs(np.asarray(got_state, np.float64)[:, 3:] - ref_state[:, 3:]) / C
    return d.max()
