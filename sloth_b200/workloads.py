"""Seeded synthetic inputs with the shapes and value ranges of the benchmark
configurations (no public dataset is involved):

* ``sinusoid_slab``   ne = n0 (1 + 0.1 sin(2 pi x / 0.5 mm)) in a 5 mm cube
* ``parabolic_trough`` ne = n0 (1 + (x / L)^2)
* ``kolmogorov_box``  mean ne0 with a Gaussian random field of 20 % RMS and a
                      k^-11/3 power spectrum from 2 pi / box to the grid Nyquist,
                      generated by FFT from a seed and clipped >= 0 (the recipe of
                      the reference's field generator, src/field_generator/
                      gaussian3D.py:215-273, normalised to an RMS instead of max|.|)
* ``gaussian_beam`` / ``lattice_beam``  rays (6, N) entering at the -z face.

Fields are float32 (nx, ny, nz) torch tensors in m^-3 on the requested device;
coordinates follow linspace(-L/2, L/2, n).
"""
from __future__ import annotations

import math

import torch

from .core.physics import C


def coords(n, L):
    return torch.linspace(-L / 2, L / 2, n, dtype=torch.float64)


def sinusoid_slab(n, *, L=5e-3, n0=1e24, period=0.5e-3, amp=0.1, device="cpu"):
    x = coords(n, L).to(device)
    prof = n0 * (1.0 + amp * torch.sin(2 * math.pi * x / period))
    return prof.to(torch.float32)[:, None, None].expand(n, n, n).contiguous()


def parabolic_trough(n, *, L=5e-3, n0=5e24, Lp=2e-3, device="cpu"):
    x = coords(n, L).to(device)
    prof = n0 * (1.0 + (x / Lp) ** 2)
    return prof.to(torch.float32)[:, None, None].expand(n, n, n).contiguous()


def kolmogorov_box(n, *, L=5e-3, mean=1e25, rms=0.2, slope=-11.0 / 3.0, seed=0, device="cpu"):
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    white = torch.randn((n, n, n), generator=g, device=device, dtype=torch.float32)
    spec = torch.fft.rfftn(white)
    h = L / (n - 1)
    kx = torch.fft.fftfreq(n, d=h, device=device) * 2 * math.pi
    kz = torch.fft.rfftfreq(n, d=h, device=device) * 2 * math.pi
    k = torch.sqrt(kx[:, None, None] ** 2 + kx[None, :, None] ** 2 + kz[None, None, :] ** 2)
    kmin, kmax = 2 * math.pi / L, math.pi / h
    band = (k >= kmin) & (k <= kmax)
    amp = torch.where(band, k.clamp_min(kmin) ** (slope / 2.0), torch.zeros_like(k))
    del k
    spec *= amp
    del amp
    field = torch.fft.irfftn(spec, s=(n, n, n))
    del spec
    field = field - field.mean()
    field *= rms / field.pow(2).mean().sqrt()
    ne = mean * (1.0 + field)
    return ne.clamp_min_(0.0).to(torch.float32).contiguous()


def gaussian_beam(N, *, waist, L=5e-3, jitter=0.0, seed=0, device="cpu", dtype=torch.float32):
    """Collimated (+z) rays with Gaussian transverse positions of 1/e^2
    intensity radius `waist` (sigma = waist/2) entering at z = -L/2; optional
    seeded angular jitter (radians, per transverse axis)."""
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    r = torch.zeros((6, N), dtype=torch.float64, device=device)
    r[0:2] = torch.randn((2, N), generator=g, device=device, dtype=torch.float64) * (waist / 2)
    r[2] = -L / 2
    _velocities(r, jitter, g)
    return r.to(dtype)


def lattice_beam(nside, *, half_width, L=5e-3, jitter=0.0, seed=0, device="cpu", dtype=torch.float32):
    """nside x nside uniform launch lattice over [-half_width, half_width]^2."""
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    t = torch.linspace(-half_width, half_width, nside, dtype=torch.float64, device=device)
    X, Y = torch.meshgrid(t, t, indexing="ij")
    N = nside * nside
    r = torch.zeros((6, N), dtype=torch.float64, device=device)
    r[0] = X.reshape(-1)
    r[1] = Y.reshape(-1)
    r[2] = -L / 2
    _velocities(r, jitter, g)
    return r.to(dtype)


def _velocities(r, jitter, g):
    N = r.shape[1]
    if jitter > 0:
        th = torch.randn((2, N), generator=g, device=r.device, dtype=torch.float64) * jitter
        sx, sy = torch.sin(th[0]), torch.sin(th[1])
        r[3] = C * sx
        r[4] = C * sy
        r[5] = C * torch.sqrt(1.0 - sx * sx - sy * sy)
    else:
        r[5] = C
