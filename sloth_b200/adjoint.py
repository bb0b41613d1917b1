"""Differentiable detector image: d(loss on the image) / d(density grid).

No counterpart in the reference, which never differentiates; the model
differentiates its ray equations (src/core/propagator.py:168-243) through a
synthetic detector image (see include/sloth_b200.h, "K4/K5"):

    image = DetectorImage.apply(ne, rays, origin, spacing, omega, spec, precision)
    loss = ((image - target) ** 2).sum()
    loss.backward()          # ne.grad from the hand-written adjoint kernels

Forward: K1 packs ne, K4 traces every ray with fixed-step Runge-Kutta-Nystrom
steps (checkpointing its state every ``spec.ckpt_every`` steps) and splats its
detector point.
Backward: K5 recomputes each checkpoint segment and runs the discrete adjoint
of the steps in reverse into d loss / d(packed grid); the pack adjoint
maps that to d loss / d ne. All on the GPU through the C ABI; there is no CPU
path.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional, Sequence, Tuple

import torch

from . import _capi as capi
from . import runtime
from .core import physics


@dataclass(frozen=True)
class DetectorSpec:
    """Detector plane, image and integration settings of the forward model."""
    window: Tuple[float, float, float, float]   # u0, u1, v0, v1 (m) on the transverse axes (ascending)
    plane: float                                # detector plane along `axis` (m)
    dtau: float                                 # step c*dt (m)
    n_px: Tuple[int, int] = (256, 256)
    axis: int = 2
    sigma_px: float = 2.0
    n_steps: int = 400
    ckpt_every: int = 20

    def params(self) -> capi.SlothImageParams:
        p = capi.SlothImageParams()
        p.dtau = float(self.dtau)
        p.n_steps = int(self.n_steps)
        p.ckpt_every = int(self.ckpt_every)
        p.probing_axis = int(self.axis)
        p.n_px[0], p.n_px[1] = int(self.n_px[0]), int(self.n_px[1])
        p.reserved = 0
        p.plane = float(self.plane)
        for k in range(4):
            p.window[k] = float(self.window[k])
        p.sigma_px = float(self.sigma_px)
        return p


def box_detector(L: float, *, n_px: int = 256, sigma_px: float = 2.0, n_steps: int = 400,
                 ckpt_every: int = 20) -> DetectorSpec:
    """Detector on the far z face of a cube [-L/2, L/2]^3 covering its cross
    section; the step is chosen so that a ray along +z crosses the cube in
    97.5% of `n_steps` steps."""
    return DetectorSpec(window=(-L / 2, L / 2, -L / 2, L / 2), plane=L / 2, dtau=L / (0.975 * n_steps),
                        n_px=(n_px, n_px), axis=2, sigma_px=sigma_px, n_steps=n_steps, ckpt_every=ckpt_every)


def _fn(name: str, precision: str):
    return getattr(capi.load(), f"{name}_{precision}")


def _image_forward(ne: torch.Tensor, rays: torch.Tensor, origin, spacing, omega: float, spec: DetectorSpec,
                   precision: str, stats: Optional[dict]):
    """K1 + K4 on this process's rays: (image, state the backward needs)."""
    if precision not in ("f32", "f64"):
        raise ValueError("precision must be 'f32' or 'f64'")
    if ne.device.type != "cuda" or rays.device.type != "cuda":
        raise ValueError("ne and rays must be CUDA tensors")
    runtime.require_device(ne.device)
    dt = torch.float32 if precision == "f32" else torch.float64
    rays = rays.to(dt).contiguous()
    if rays.dim() != 2 or rays.shape[0] != 6:
        raise ValueError("rays must be (6, N)")
    grid = runtime.pack_grid(ne.detach(), origin, spacing, omega, precision=precision, device=ne.device,
                             layout="values")
    params = spec.params()
    n = int(rays.shape[1])
    ws_bytes = int(capi.load().sloth_image_workspace_bytes(ctypes.byref(params), n))
    if ws_bytes == 0:
        raise ValueError("invalid detector spec")
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=ne.device)
    image = torch.empty(tuple(spec.n_px), dtype=dt, device=ne.device)
    steps = None
    if stats is not None:
        steps = torch.zeros(1, dtype=torch.int64, device=ne.device)
        stats["ray_steps"] = steps
    stream = torch.cuda.current_stream(ne.device).cuda_stream
    capi.check(_fn("sloth_image_forward", precision)(grid.desc, capi.ptr(grid.data), ctypes.byref(params),
                                                     capi.ptr(rays), n, capi.ptr(image),
                                                     capi.ptr(steps) if steps is not None else None,
                                                     capi.ptr(ws), ws_bytes, stream), "sloth_image_forward")
    # the workspace's ray order refers to `rays`, which the state keeps alive
    state = dict(grid=grid, ws=ws, ws_bytes=ws_bytes, params=params, n=n, precision=precision,
                 ne_dtype=ne.dtype, ne_shape=tuple(ne.shape), rays=rays)
    return image, state


def _image_backward(state: dict, grad_image: torch.Tensor) -> torch.Tensor:
    """K5 + the pack adjoint: d loss / d ne from this process's rays."""
    grid, precision = state["grid"], state["precision"]
    dt = torch.float32 if precision == "f32" else torch.float64
    gi = grad_image.to(dt).contiguous()
    gg = torch.empty_like(grid.data)
    stream = torch.cuda.current_stream(gi.device).cuda_stream
    capi.check(_fn("sloth_image_backward", precision)(grid.desc, capi.ptr(grid.data), ctypes.byref(state["params"]),
                                                      state["n"], capi.ptr(gi), capi.ptr(gg), capi.ptr(state["ws"]),
                                                      state["ws_bytes"], stream), "sloth_image_backward")
    ne_grad = torch.empty(state["ne_shape"], dtype=dt, device=gi.device)
    capi.check(_fn("sloth_grid_pack_adjoint", precision)(grid.desc, capi.ptr(gg), 1.0 / grid.nc,
                                                         capi.ptr(ne_grad), stream), "sloth_grid_pack_adjoint")
    return ne_grad.to(state["ne_dtype"])


def _sum_over(t: torch.Tensor, group) -> torch.Tensor:
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.SUM, group=group)
    return t


class DetectorImage(torch.autograd.Function):
    """image = F(ne): differentiable with respect to ne only.

    With a process group, the rays are sharded over its ranks (each passes
    its own) and the image is the sum over ranks, so every rank returns the
    image of all rays. The backward then needs the same d loss / d image on
    every rank (a loss computed from the summed image), and returns d loss /
    d ne summed over ranks: the gradient of all rays on every rank. These are
    the model's only exchanges, one all-reduce each way (an image and a grid);
    every rank must take part in both."""

    @staticmethod
    def forward(ctx, ne: torch.Tensor, rays: torch.Tensor, origin: Sequence[float], spacing: Sequence[float],
                omega: float, spec: DetectorSpec, precision: str = "f32", stats: Optional[dict] = None,
                group=None):
        image, state = _image_forward(ne, rays, origin, spacing, omega, spec, precision, stats)
        ctx.state, ctx.group = state, group
        if group is not None:
            _sum_over(image, group)
        return image

    @staticmethod
    def backward(ctx, grad_image: torch.Tensor):
        ne_grad = _image_backward(ctx.state, grad_image)
        if ctx.group is not None:
            _sum_over(ne_grad, ctx.group)
        return ne_grad, None, None, None, None, None, None, None, None


def detector_image(ne: torch.Tensor, rays: torch.Tensor, spec: DetectorSpec, *, origin, spacing,
                   lwl: Optional[float] = None, omega: Optional[float] = None,
                   precision: str = "f32", stats: Optional[dict] = None, group=None) -> torch.Tensor:
    """The detector image of `rays` (6, N) through the density `ne` (m^-3);
    differentiable with respect to `ne`. If `stats` is a dict, its
    "ray_steps" entry receives a device counter of the steps taken (this
    process's rays). With a torch.distributed process group, each rank passes
    its share of the rays and gets the image and the gradient of all of them
    (see DetectorImage)."""
    if omega is None:
        if lwl is None:
            raise ValueError("give lwl or omega")
        omega = physics.omega_of(lwl)
    return DetectorImage.apply(ne, rays, tuple(map(float, origin)), tuple(map(float, spacing)), float(omega),
                               spec, precision, stats, group)


def image_loss_grad(ne: torch.Tensor, rays: torch.Tensor, target: torch.Tensor, spec: DetectorSpec, *, origin,
                    spacing, lwl: float, precision: str = "f32", group=None):
    """L = ||I(ne) - target||^2 and dL/dne (same dtype as ne); with a process
    group, over the rays of all its ranks (the same L and dL/dne on each)."""
    x = ne.detach().requires_grad_(True)
    img = detector_image(x, rays, spec, origin=origin, spacing=spacing, lwl=lwl, precision=precision,
                         group=group)
    loss = (img.to(torch.float64) - target.to(torch.float64)).pow(2).sum()
    loss.backward()
    return float(loss.detach()), x.grad
