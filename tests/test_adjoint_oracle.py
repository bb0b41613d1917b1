"""CPU checks of the detector-image oracle (oracle/adjoint_torch.py), the
reference the adjoint kernels are tested against: its steps equal the tracer
oracle's (which is pinned to the reference's golden vectors) away from the
faces, it integrates a linear density ramp exactly, and its autograd
gradient equals its own central differences."""
import math

import numpy as np
import torch

from oracle import adjoint_torch as at
from oracle import ref_restated as rr
from sloth_b200 import workloads
from sloth_b200.core import physics

L = 5e-3
LWL = 532e-9


def test_steps_match_the_tracer_oracle_inside_the_grid():
    """The detector model steps like the tracer oracle (which is pinned to the
    reference's golden vectors): on rays that stay inside the grid, their
    states agree to rounding."""
    n = 20
    h = L / (n - 1)
    ne = workloads.kolmogorov_box(n, L=L, mean=2e26, rms=0.3, seed=4).double()
    om = physics.omega_of(LWL)
    # rays that start deep inside and stay there for 12 steps
    g = torch.Generator().manual_seed(1)
    rays = torch.zeros(6, 64, dtype=torch.float64)
    rays[0:3] = (torch.rand(3, 64, generator=g, dtype=torch.float64) - 0.5) * (0.4 * L)
    d = torch.randn(3, 64, generator=g, dtype=torch.float64)
    rays[3:6] = d / d.norm(dim=0) * at.C
    dtau, steps = h / 2, 12
    p, w, taken = at.final_states(ne, (-L / 2,) * 3, (h,) * 3, om, rays, dtau=dtau, n_steps=steps)
    assert int(taken.min()) == steps
    grid = rr.Grid(ne.numpy(), (-L / 2,) * 3, (h,) * 3, om)
    ref = rr.trace_rays(grid, rays.numpy(), dtau=dtau, first_save=steps, save_every=1, n_saves=1)["state"][0]
    pos = p.numpy().T * h - L / 2
    vel = w.numpy().T * at.C * h / dtau
    np.testing.assert_allclose(pos, ref[:3], rtol=0, atol=1e-13 * L)
    np.testing.assert_allclose(vel, ref[3:], rtol=1e-11, atol=1e-6)


def test_linear_ramp_is_integrated_exactly():
    # ne = n0 (1 + x/Lr): constant gradient, so the step reproduces the parabola
    n, n0, Lr = 24, 1e26, 2e-3
    h = L / (n - 1)
    x = -L / 2 + h * torch.arange(n, dtype=torch.float64)
    ne = (n0 * (1 + x / Lr))[:, None, None].expand(n, n, n).contiguous()
    om = physics.omega_of(LWL)
    rays = torch.zeros(6, 5, dtype=torch.float64)
    rays[0] = torch.linspace(-1e-3, 1e-3, 5, dtype=torch.float64)
    rays[2] = -L / 2
    rays[5] = at.C
    dtau, T = h / 3, 30                     # stays inside: 30 steps of h/3 = 10 cells
    p, w, _ = at.final_states(ne, (-L / 2,) * 3, (h,) * 3, om, rays, dtau=dtau, n_steps=T)
    nc = physics.critical_density(om)
    a = -0.5 * at.C ** 2 * (n0 / nc) / Lr          # d^2 x / dt^2 (m/s^2)
    t = T * dtau / at.C
    np.testing.assert_allclose(p[:, 0].numpy() * h - L / 2, rays[0].numpy() + 0.5 * a * t * t, rtol=0, atol=1e-15)
    np.testing.assert_allclose(w[:, 0].numpy() * at.C * h / dtau, a * t, rtol=1e-12)
    np.testing.assert_allclose(p[:, 2].numpy() * h - L / 2, -L / 2 + T * dtau, rtol=0, atol=1e-15)
    # the image of the projected points is their splat
    plane = 0.0
    img = at.detector_image(ne, (-L / 2,) * 3, (h,) * 3, om, rays, dtau=dtau, n_steps=T, plane=plane,
                            window=(-L / 2, L / 2, -L / 2, L / 2), n_px=(40, 40), sigma_px=1.5)
    X = p[:, 0] + (plane + L / 2 - p[:, 2] * h) / h * (w[:, 0] / w[:, 2])
    a_px = (X * h) / (L / 40) - 0.5
    b_px = torch.full_like(a_px, (L / 2) / (L / 40) - 0.5)
    gi = at.splat_profile(torch.arange(40, dtype=torch.float64)[None] - a_px[:, None], 1.5)
    gj = at.splat_profile(torch.arange(40, dtype=torch.float64)[None] - b_px[:, None], 1.5)
    np.testing.assert_allclose(img.numpy(), (gi.T @ gj).numpy() / (2 * math.pi * 1.5 ** 2), rtol=1e-12, atol=1e-15)
    assert abs(float(img.sum()) - 5.0) < 0.02        # every ray deposits ~1 (the taper trims < 0.3%)


def test_oracle_autograd_matches_its_central_differences():
    n = 12
    h = L / (n - 1)
    om = physics.omega_of(LWL)
    ne0 = workloads.kolmogorov_box(n, L=L, mean=3e26, rms=0.3, seed=7).double()
    ne1 = workloads.kolmogorov_box(n, L=L, mean=3e26, rms=0.3, seed=8).double()
    rays = workloads.gaussian_beam(400, waist=2e-3, L=L, seed=3, jitter=3e-3).double()
    kw = dict(dtau=L / (0.975 * 40), n_steps=40, plane=L / 2, window=(-L / 2, L / 2, -L / 2, L / 2),
              n_px=(16, 16), sigma_px=1.2)
    target = at.detector_image(ne0, (-L / 2,) * 3, (h,) * 3, om, rays, **kw)

    def loss(ne):
        return ((at.detector_image(ne, (-L / 2,) * 3, (h,) * 3, om, rays, **kw) - target) ** 2).sum()

    x = ne1.clone().requires_grad_(True)
    loss(x).backward()
    g = x.grad
    assert torch.isfinite(g).all() and float(g.abs().max()) > 0
    rng = np.random.default_rng(0)
    idx = [tuple(int(v) for v in rng.integers(2, n - 2, 3)) for _ in range(6)]
    idx.append(tuple(int(v) for v in torch.nonzero(g.abs() == g.abs().max())[0]))
    for i in idx:
        eps = 1e-4 * float(ne1[i])
        a, b = ne1.clone(), ne1.clone()
        a[i] += eps
        b[i] -= eps
        fd = (float(loss(a)) - float(loss(b))) / (2 * eps)
        assert abs(fd - float(g[i])) <= 1e-5 * float(g.abs().max()) + 1e-4 * abs(fd), (i, fd, float(g[i]))
