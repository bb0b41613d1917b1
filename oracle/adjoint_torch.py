"""Test infrastructure only: a CPU FP64 restatement of the detector-image
forward model, differentiable with torch autograd. It stands in for jax.grad
of the reference, which cannot run here because JAX is not installed. The
device kernels are checked against it; the product never imports it.

The model, in the tracers' scaled units (positions in grid cells, velocity
in cells per step, one step = unit step):
  * pack: q = ne * (1/nc); the gradient channels are dq/du per cell along each
    axis, central inside and one-sided on the faces. This is jnp.gradient
    with coordinates, as in precompute_gradients
    (src/core/propagator.py:72-93), times h.
  * RHS: dw/dstep = S * interp(dq/du)(p), S = -(dtau/h)^2 / 2; trilinear
    interpolation with cell i = floor(p) clamped to [0, n-2] and fill 0
    outside [0, n-1] (src/core/interpolator.py:79-104). This is dv/dt in
    dsdt (src/core/propagator.py:168-243) in scaled form.
  * fixed-step fourth-order Runge-Kutta-Nystrom steps (the tracers' method:
    stages at p, p + w/2 + A1/8, p + w + A2/2; p' = p + w + (A1 + 2 A2)/6,
    w' = w + (A1 + 4 A2 + A3)/6), at most n_steps. A ray stops once it is outside the
    grid on some axis and moving away from it along that axis; the check
    runs before each step.
  * straight line to the detector plane (src/shared/propagation.py:92-134);
    Gaussian splat with a C2 taper between 3 and 4 sigma, 1/(2 pi sigma^2)
    per ray.
"""
from __future__ import annotations

import math

import torch

ALPHA = 3.14207787e-4          # nc = ALPHA * omega^2 (src/core/propagator.py:73)
C = 299792458.0


def pack_channels(ne: torch.Tensor, scale: float) -> torch.Tensor:
    """(3, nx, ny, nz) gradient channels dq/du_k per cell, q = ne * scale."""
    q = ne * scale
    out = []
    for ax in range(3):
        n = q.shape[ax]
        lo = q.narrow(ax, 1, 1) - q.narrow(ax, 0, 1)
        hi = q.narrow(ax, n - 1, 1) - q.narrow(ax, n - 2, 1)
        parts = [lo]
        if n > 2:
            parts.append(0.5 * (q.narrow(ax, 2, n - 2) - q.narrow(ax, 0, n - 2)))
        parts.append(hi)
        out.append(torch.cat(parts, dim=ax))
    return torch.stack(out)


def interp(ch: torch.Tensor, p: torch.Tensor) -> torch.Tensor:
    """Trilinear interpolation of the (3, nx, ny, nz) channels at p (N, 3)
    cells, 0 outside; returns (N, 3)."""
    n = ch.shape[1:]
    lim = torch.tensor([k - 1 for k in n], dtype=p.dtype)
    inside = ((p >= 0) & (p <= lim)).all(dim=1)
    # points outside take the fill value; zero them first so that no NaN or
    # out-of-range index reaches the gather (or its gradient)
    p = torch.where(inside[:, None], p, torch.zeros_like(p))
    i = torch.minimum(torch.floor(p.detach()), lim - 1).to(torch.long)
    f = p - i.to(p.dtype)
    flat = ch.reshape(3, -1)
    sx, sy = n[1] * n[2], n[2]
    base = i[:, 0] * sx + i[:, 1] * sy + i[:, 2]
    acc = torch.zeros(p.shape[0], 3, dtype=p.dtype)
    for dx in (0, 1):
        wx = f[:, 0] if dx else 1 - f[:, 0]
        for dy in (0, 1):
            wy = f[:, 1] if dy else 1 - f[:, 1]
            for dz in (0, 1):
                wz = f[:, 2] if dz else 1 - f[:, 2]
                idx = base + dx * sx + dy * sy + dz
                acc = acc + (wx * wy * wz)[:, None] * flat[:, idx].T
    return torch.where(inside[:, None], acc, torch.zeros_like(acc))


def gone(p: torch.Tensor, w: torch.Tensor, lim: torch.Tensor) -> torch.Tensor:
    out = ((p < 0) & (w <= 0)) | ((p > lim) & (w >= 0)) | ~torch.isfinite(p) | ~torch.isfinite(w)
    return out.any(dim=1)


def splat_profile(d: torch.Tensor, sigma: float) -> torch.Tensor:
    u = d.abs() / sigma
    x = u - 3.0
    taper = torch.where(u <= 3.0, torch.ones_like(u), 1.0 - x ** 3 * (10.0 - 15.0 * x + 6.0 * x ** 2))
    g = torch.exp(-0.5 * (d / sigma) ** 2) * taper
    return torch.where(u >= 4.0, torch.zeros_like(g), g)


def final_states(ne, origin, spacing, omega, rays, *, dtau, n_steps):
    """The steps of every ray; returns (p, w) (N, 3) in cells, cells per step, and
    the steps taken."""
    ne = ne.to(torch.float64)
    rays = torch.as_tensor(rays, dtype=torch.float64)
    h = torch.tensor(spacing, dtype=torch.float64)
    o = torch.tensor(origin, dtype=torch.float64)
    ch = pack_channels(ne, 1.0 / (ALPHA * omega ** 2))
    S = -0.5 * (dtau / h) ** 2
    p = ((rays[0:3].T - o) / h).clone()
    w = rays[3:6].T * (dtau / h) / C
    lim = torch.tensor([k - 1 for k in ne.shape], dtype=torch.float64)
    alive = torch.ones(p.shape[0], dtype=torch.bool)
    steps = torch.zeros(p.shape[0], dtype=torch.long)
    for _ in range(n_steps):
        alive = alive & ~gone(p.detach(), w.detach(), lim)
        if not bool(alive.any()):
            break
        A1 = S * interp(ch, p)
        A2 = S * interp(ch, p + 0.5 * w + 0.125 * A1)
        A3 = S * interp(ch, p + w + 0.5 * A2)
        pn = p + w + (A1 + 2.0 * A2) / 6.0
        wn = w + (A1 + 4.0 * A2 + A3) / 6.0
        m = alive[:, None]
        p = torch.where(m, pn, p)
        w = torch.where(m, wn, w)
        steps = steps + alive.to(torch.long)
    return p, w, steps


def detector_image(ne, origin, spacing, omega, rays, *, dtau, n_steps, axis=2, plane, window, n_px, sigma_px):
    """The image (n_px[0], n_px[1]) as a differentiable function of ne."""
    p, w, _ = final_states(ne, origin, spacing, omega, rays, dtau=dtau, n_steps=n_steps)
    t1 = 1 if axis == 0 else 0
    t2 = 1 if axis == 2 else 2
    pc = (plane - origin[axis]) / spacing[axis]
    wa = w[:, axis]
    ok = (wa != 0) & torch.isfinite(wa)
    safe = torch.where(ok, wa, torch.ones_like(wa))
    t = (pc - p[:, axis]) / safe
    coords = []
    for d, ax in enumerate((t1, t2)):
        lo, hi = window[2 * d], window[2 * d + 1]
        pix = (hi - lo) / n_px[d]
        X = p[:, ax] + t * w[:, ax]
        coords.append((origin[ax] - lo) / pix - 0.5 + (spacing[ax] / pix) * X)
    a, b = coords
    ok = ok & torch.isfinite(a) & torch.isfinite(b)
    a = torch.where(ok, a, torch.full_like(a, -1e6))
    b = torch.where(ok, b, torch.full_like(b, -1e6))
    gi = splat_profile(torch.arange(n_px[0], dtype=torch.float64)[None, :] - a[:, None], sigma_px)
    gj = splat_profile(torch.arange(n_px[1], dtype=torch.float64)[None, :] - b[:, None], sigma_px)
    gi = gi * ok[:, None].to(gi.dtype)
    return (gi.T @ gj) / (2.0 * math.pi * sigma_px ** 2)
