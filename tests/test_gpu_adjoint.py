"""Detector image and its adjoint on the GPU, through the C ABI: the image and
d loss / d ne against the torch FP64 autograd oracle, the pack adjoint
against its defining identity, checkpoint-length invariance, error codes,
and d loss / d ne against central finite differences on the 128^3 /
1e6-ray / 400-step workload."""
import ctypes
import math

import numpy as np
import pytest
import torch

from oracle import adjoint_torch as at
from sloth_b200 import _capi, adjoint, runtime, workloads
from sloth_b200.core import physics

pytestmark = pytest.mark.gpu

L = 5e-3
LWL = 532e-9
OM = physics.omega_of(LWL)


def _small(n=24, nrays=3000, steps=60, ckpt=7, npx=32, sigma=1.5):
    h = L / (n - 1)
    ne0 = workloads.kolmogorov_box(n, L=L, mean=2e26, rms=0.3, seed=11).double()
    ne1 = workloads.kolmogorov_box(n, L=L, mean=2e26, rms=0.3, seed=12).double()
    rays = workloads.gaussian_beam(nrays, waist=2e-3, L=L, seed=5, jitter=2e-3).double()
    spec = adjoint.DetectorSpec(window=(-L / 2, L / 2, -L / 2, L / 2), plane=L / 2, dtau=L / (0.975 * steps),
                                n_px=(npx, npx), sigma_px=sigma, n_steps=steps, ckpt_every=ckpt)
    return h, ne0, ne1, rays, spec


def _oracle(ne, rays, h, spec):
    return at.detector_image(ne, (-L / 2,) * 3, (h,) * 3, OM, rays, dtau=spec.dtau, n_steps=spec.n_steps,
                             axis=spec.axis, plane=spec.plane, window=spec.window, n_px=spec.n_px,
                             sigma_px=spec.sigma_px)


def _oracle_grad(ne, rays, target, h, spec):
    x = ne.clone().requires_grad_(True)
    loss = ((_oracle(x, rays, h, spec) - target) ** 2).sum()
    loss.backward()
    return float(loss.detach()), x.grad


def _kernel(ne, rays, h, spec, precision, target=None):
    dt = torch.float32 if precision == "f32" else torch.float64
    x = ne.to("cuda", dt).requires_grad_(True)
    img = adjoint.detector_image(x, rays.to("cuda", dt), spec, origin=(-L / 2,) * 3, spacing=(h,) * 3, omega=OM,
                                 precision=precision)
    if target is None:
        return img.detach().double().cpu(), None
    loss = (img.double() - target.to("cuda")).pow(2).sum()
    loss.backward()
    return img.detach().double().cpu(), x.grad.double().cpu()


def _rel(a, b):
    return float((a - b).abs().max() / b.abs().max())


def test_image_and_gradient_f64_match_oracle():
    h, ne0, ne1, rays, spec = _small()
    target = _oracle(ne0, rays, h, spec).detach()
    img_o = _oracle(ne1, rays, h, spec).detach()
    _, g_o = _oracle_grad(ne1, rays, target, h, spec)
    img, g = _kernel(ne1, rays, h, spec, "f64", target)
    assert float(img.sum()) > 0.5 * rays.shape[1]
    assert _rel(img, img_o) < 1e-11
    assert _rel(g, g_o) < 1e-9, _rel(g, g_o)


def test_image_and_gradient_f32_match_oracle():
    h, ne0, ne1, rays, spec = _small()
    target = _oracle(ne0, rays, h, spec).detach()
    img_o = _oracle(ne1, rays, h, spec).detach()
    _, g_o = _oracle_grad(ne1, rays, target, h, spec)
    img, g = _kernel(ne1, rays, h, spec, "f32", target)
    assert _rel(img, img_o) < 2e-5
    # FP32 gradient: max error 1e-3 of the largest component, and the field
    # as a whole to 1e-4 in the L2 sense
    assert _rel(g, g_o) < 1e-3, _rel(g, g_o)
    assert float((g - g_o).norm() / g_o.norm()) < 1e-4


@pytest.mark.parametrize("precision,tol", [("f64", 1e-11), ("f32", 2e-5)])
def test_image_with_tiled_and_direct_splats(precision, tol):
    # A CTA splats the rays whose windows fit a 32 x 32 pixel tile in shared
    # memory and the others directly. On a 96 x 96 detector, 256 rays from
    # about 50 entry cells spread their windows over more than one tile, so
    # both paths run in the same CTAs; the image must equal the oracle's.
    h, _, ne1, rays, spec = _small()
    spec = adjoint.DetectorSpec(window=spec.window, plane=spec.plane, dtau=spec.dtau, n_px=(96, 96),
                                sigma_px=spec.sigma_px, n_steps=spec.n_steps, ckpt_every=spec.ckpt_every)
    img_o = _oracle(ne1, rays, h, spec).detach()
    img, _ = _kernel(ne1, rays, h, spec, precision)
    assert float(img.sum()) > 0.5 * rays.shape[1]
    assert _rel(img, img_o) < tol


def test_gradient_independent_of_checkpoint_length():
    h, ne0, ne1, rays, _ = _small()
    grads = []
    for ck in (1, 13, 32):
        spec = adjoint.DetectorSpec(window=(-L / 2, L / 2, -L / 2, L / 2), plane=L / 2, dtau=L / (0.975 * 60),
                                    n_px=(32, 32), sigma_px=1.5, n_steps=60, ckpt_every=ck)
        target = _kernel(ne0, rays, h, spec, "f64")[0]
        grads.append(_kernel(ne1, rays, h, spec, "f64", target)[1])
    for g in grads[1:]:
        assert _rel(g, grads[0]) < 1e-12


def test_pack_adjoint_is_the_transpose_of_pack():
    # <pack(ne), G> = <ne, pack_adjoint(G)> for random ne and G
    n = (9, 7, 11)
    desc = _capi.grid_desc(n, (0.0, 0.0, 0.0), (1e-4, 2e-4, 3e-4))
    lib = _capi.load()
    gen = torch.Generator().manual_seed(3)
    ne = torch.randn(n, generator=gen, dtype=torch.float64).cuda()
    G = torch.randn(int(np.prod(n)) * 4, generator=gen, dtype=torch.float64).cuda()
    packed = torch.empty_like(G)
    scale = 0.37
    _capi.check(lib.sloth_grid_pack_f64(desc, _capi.ptr(ne), 1, scale, _capi.ptr(packed), None))
    back = torch.empty(n, dtype=torch.float64, device="cuda")
    _capi.check(lib.sloth_grid_pack_adjoint_f64(desc, _capi.ptr(G), scale, _capi.ptr(back), None))
    lhs = float((packed * G).sum())
    rhs = float((ne * back).sum())
    assert abs(lhs - rhs) <= 1e-12 * (packed.abs() * G.abs()).sum().item()
    G32 = G.float()
    back32 = torch.empty(n, dtype=torch.float32, device="cuda")
    _capi.check(lib.sloth_grid_pack_adjoint_f32(desc, _capi.ptr(G32), scale, _capi.ptr(back32), None))
    np.testing.assert_allclose(back32.double().cpu().numpy(), back.cpu().numpy(), rtol=1e-5, atol=1e-6)


def test_error_codes():
    lib = _capi.load()
    h, _, ne1, rays, spec = _small(n=8, nrays=10)
    g = runtime.pack_grid(ne1.cuda(), (-L / 2,) * 3, (h,) * 3, OM, precision="f32")
    r = rays.float().cuda()
    img = torch.empty(spec.n_px, device="cuda")
    p = spec.params()
    ws_bytes = lib.sloth_image_workspace_bytes(ctypes.byref(p), 10)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    fwd = lambda prm, wsb=ws_bytes: lib.sloth_image_forward_f32(g.desc, _capi.ptr(g.data), ctypes.byref(prm),
                                                               _capi.ptr(r), 10, _capi.ptr(img), None,
                                                               _capi.ptr(ws), wsb, None)
    assert fwd(p) == _capi.SLOTH_OK
    assert fwd(p, ws_bytes - 1) == _capi.SLOTH_ERR_WORKSPACE_TOO_SMALL
    for field, bad in (("ckpt_every", 0), ("ckpt_every", 33), ("sigma_px", 0.0), ("sigma_px", 9.0),
                       ("n_steps", 0), ("probing_axis", 3), ("reserved", 1), ("dtau", -1.0)):
        q = spec.params()
        setattr(q, field, bad)
        assert fwd(q) == _capi.SLOTH_ERR_INVALID_ARGUMENT, field
    q = spec.params()
    q.window[1] = q.window[0]
    assert fwd(q) == _capi.SLOTH_ERR_INVALID_ARGUMENT
    assert lib.sloth_image_forward_f32(g.desc, None, ctypes.byref(p), _capi.ptr(r), 10, _capi.ptr(img), None,
                                       _capi.ptr(ws), ws_bytes, None) == _capi.SLOTH_ERR_NULL_POINTER
    torch.cuda.synchronize()


def test_gradient_against_finite_differences_128cube_1e6_rays():
    """The 128^3 FP32 grid, 1e6 rays, 400 fourth-order steps (the tracer's
    Runge-Kutta-Nystrom step) with checkpoints every
    20, 256^2 image with a 2-pixel splat: d L / d ne from the FP32 adjoint
    against central differences of the FP64 forward at 64 random voxels of
    the beam's core."""
    n, nrays = 128, 1_000_000
    h = L / (n - 1)
    spec = adjoint.box_detector(L, n_px=256, sigma_px=2.0, n_steps=400, ckpt_every=20)
    ne_t = workloads.kolmogorov_box(n, L=L, mean=1e25, rms=0.2, seed=41, device="cuda")
    ne = workloads.kolmogorov_box(n, L=L, mean=1e25, rms=0.2, seed=42, device="cuda")
    rays = workloads.gaussian_beam(nrays, waist=1.5e-3, L=L, seed=43, device="cuda")
    kw = dict(origin=(-L / 2,) * 3, spacing=(h,) * 3, lwl=LWL)
    with torch.no_grad():
        target = adjoint.detector_image(ne_t, rays, spec, **kw, precision="f64").double()
    loss32, g32 = adjoint.image_loss_grad(ne, rays, target, spec, **kw, precision="f32")
    loss64, g64 = adjoint.image_loss_grad(ne.double(), rays.double(), target, spec, **kw, precision="f64")
    assert abs(loss32 - loss64) < 1e-4 * loss64
    rng = np.random.default_rng(7)
    c = n // 2
    vox = [tuple(int(v) for v in rng.integers(c - 30, c + 30, 3)) for _ in range(64)]
    ne64 = ne.double()
    r64 = rays.double()

    def loss_at(x):
        with torch.no_grad():
            img = adjoint.detector_image(x, r64, spec, **kw, precision="f64")
        return float((img - target).pow(2).sum())

    fd = []
    for v in vox:
        eps = 1e-3 * float(ne64[v])
        x = ne64.clone()
        x[v] += eps
        lp = loss_at(x)
        x[v] -= 2 * eps
        lm = loss_at(x)
        fd.append((lp - lm) / (2 * eps))
    fd = np.array(fd)
    a64 = np.array([float(g64[v]) for v in vox])
    a32 = np.array([float(g32[v]) for v in vox])
    scale = np.abs(fd).max()
    assert scale > 0
    # FP64 adjoint vs FP64 central differences (O(eps^2) truncation)
    assert np.abs(a64 - fd).max() <= 1e-3 * scale, np.abs(a64 - fd).max() / scale
    # FP32 adjoint vs the same differences
    assert np.abs(a32 - fd).max() <= 1e-2 * scale, np.abs(a32 - fd).max() / scale
    # the whole FP32 gradient against the FP64 one
    assert float((g32.double() - g64).norm() / g64.norm()) < 1e-2


def test_process_group_of_one_matches_the_local_model():
    """With a process group (NCCL, here one rank) the image and the gradient
    pass through an all-reduce each; over one rank they must equal the local
    model's, up to the order of the splat and gradient atomics."""
    import datetime
    import socket

    import torch.distributed as dist
    h, ne0, ne1, rays, spec = _small()
    target = _kernel(ne1, rays, h, spec, "f64")[0]
    img, grad = _kernel(ne0, rays, h, spec, "f64", target)
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60), device_id=torch.device("cuda", 0))
    try:
        x = ne0.to("cuda").requires_grad_(True)
        img_g = adjoint.detector_image(x, rays.to("cuda"), spec, origin=(-L / 2,) * 3, spacing=(h,) * 3, omega=OM,
                                       precision="f64", group=dist.group.WORLD)
        (img_g.double() - target.to("cuda")).pow(2).sum().backward()
        torch.cuda.synchronize()
        assert _rel(img_g.detach().cpu(), img) < 1e-12
        assert _rel(x.grad.cpu(), grad) < 1e-12
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_no_rays_give_a_zero_image_and_gradient(precision):
    """Zero rays: the image is all zeros, and so is d loss / d ne, of the
    grid's shape, for any target."""
    h, _, ne1, _, spec = _small()
    rays = torch.zeros((6, 0), dtype=torch.float64)
    target = torch.rand(tuple(spec.n_px), dtype=torch.float64)
    img, g = _kernel(ne1, rays, h, spec, precision, target)
    assert img.shape == tuple(spec.n_px) and not img.any()
    assert g.shape == ne1.shape and not g.any()
