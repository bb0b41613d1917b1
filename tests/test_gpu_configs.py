"""Parity at the sizes of the two small workload configurations, through the
C ABI, against the oracle:

* the 128^3 sinusoidal slab with 1e4 Gaussian-beam rays (the whole
  configuration);
* the 256^3 parabolic trough with rays of its 1000 x 1000 jittered launch
  lattice. The grid is the configuration's; the rays are every 50th lattice
  ray, so that the FP64 oracle finishes in seconds;
* a 128^3 Kolmogorov box with inverse bremsstrahlung, the headline mode at
  a size the oracle can follow;
* 40 saves a few steps apart, which the tracer's interior runs must stop at.

The trough also has an analytic answer: its transverse motion is simple
harmonic, x(t) = x0 cos(W t) + (vx0 / W) sin(W t) with W = c sqrt(n0/nc) / Lp,
and its packed gradient and trilinear interpolation are exact inside the outer
cells (central differences of a quadratic, interpolation of a linear
function). So a mid-box save is also checked against x(t)."""
import numpy as np
import pytest
import torch

from helpers import C, direction_error, position_error, run_kernel, run_oracle
from sloth_b200 import runtime, workloads

pytestmark = pytest.mark.gpu

L = 5e-3
LWL = 532e-9
OMEGA = 2 * np.pi * C / LWL


def _tol(precision):
    return 1e-10 if precision == "f64" else 1e-6


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_config_sinusoid_slab_128_1e4_rays(precision):
    n = 128
    h = L / (n - 1)
    ne = workloads.sinusoid_slab(n, L=L, n0=1e24).double().numpy()
    rays = workloads.gaussian_beam(10_000, waist=1e-3, L=L, seed=101).numpy()
    sched = runtime.schedule_times(np.array([np.sqrt(8.0) * L]), (h, h, h))
    kw = dict(project=True, plane=L / 2)
    k = run_kernel(ne, rays, (-L / 2,) * 3, (h,) * 3, OMEGA, sched, precision=precision, **kw)
    o = run_oracle(ne, rays, (-L / 2,) * 3, (h,) * 3, OMEGA, sched, **kw)
    assert position_error(k["state"], o["state"], L) < _tol(precision)
    assert direction_error(k["state"], o["state"]) < _tol(precision)
    ph = np.abs(o["phase"]).max()
    assert np.abs(k["phase"] - o["phase"]).max() <= _tol(precision) * ph
    assert (k["status"] != o["status"]).mean() < 1e-3
    assert (k["steps"] != o["steps"]).mean() < 1e-3


@pytest.mark.parametrize("integ", ["rkn", "rk4"])
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_config_trough_256_lattice(precision, integ):
    n, n0, Lp = 256, 5e24, 2e-3
    h = L / (n - 1)
    # the quadratic in FP64: differences of float32-rounded densities would
    # add acceleration noise near x = 0 at the 1e-10 L level
    x = np.linspace(-L / 2, L / 2, n)
    ne = np.ascontiguousarray(np.broadcast_to((n0 * (1.0 + (x / Lp) ** 2))[:, None, None], (n, n, n)))
    lattice = workloads.lattice_beam(1000, half_width=L / 2 - h, L=L, jitter=1e-3, seed=7, dtype=torch.float64)
    rays64 = lattice[:, ::50].contiguous().numpy()
    rays = rays64.astype(np.float32)
    tau_mid = 0.5 * L
    sched = runtime.schedule_times(np.array([tau_mid]), (h, h, h))
    k = run_kernel(ne, rays, (-L / 2,) * 3, (h,) * 3, OMEGA, sched, precision=precision, integrator=integ)
    o = run_oracle(ne, rays, (-L / 2,) * 3, (h,) * 3, OMEGA, sched, integrator=integ)
    assert position_error(k["state"], o["state"], L) < _tol(precision)
    assert direction_error(k["state"], o["state"]) < _tol(precision)
    # analytic x(t) for rays that stay out of the outer cells, at the
    # schedule's own save time (c t = first_save * dtau)
    nc = 3.14207787e-4 * OMEGA ** 2
    W = C * np.sqrt(n0 / nc) / Lp
    t = sched.first_save * sched.dtau / C
    x0 = rays.astype(np.float64)[0]
    vx0 = rays.astype(np.float64)[3]
    x_an = x0 * np.cos(W * t) + (vx0 / W) * np.sin(W * t)
    inner = np.abs(x0) < L / 2 - 3 * h
    assert inner.sum() > 10_000
    dx = np.abs(k["state"][-1][0].astype(np.float64) - x_an)[inner].max() / L
    assert dx < (1e-9 if precision == "f64" else 1e-6), dx


@pytest.mark.parametrize("integ", ["rkn", "rk4"])
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_kolmogorov_128_with_absorption(precision, integ):
    """The headline mode at a size where interior runs are long: a 128^3
    Kolmogorov box (20% RMS), inverse bremsstrahlung at Te = 20 eV, Z = 1,
    2e4 rays of a 3 mm beam, three saves; against the oracle, with either
    integrator (Runge-Kutta-Nystrom, or the classical RK4 the workload
    descriptions name)."""
    n = 128
    h = L / (n - 1)
    ne = workloads.kolmogorov_box(n, L=L, mean=1e25, rms=0.2, seed=31).numpy()
    rays = workloads.gaussian_beam(20_000, waist=1.5e-3, L=L, seed=32).numpy()
    sched = runtime.schedule_times(np.linspace(0.0, L, 3), (h, h, h))
    kw = dict(project=True, plane=L / 2, inv_brems=True, Te=20.0, Z=1.0, integrator=integ)
    k = run_kernel(ne, rays, (-L / 2,) * 3, (h,) * 3, OMEGA, sched, precision=precision, **kw)
    o = run_oracle(ne, rays, (-L / 2,) * 3, (h,) * 3, OMEGA, sched, **kw)
    assert position_error(k["state"], o["state"], L) < _tol(precision)
    assert direction_error(k["state"], o["state"]) < _tol(precision)
    side = (np.abs(o["state"][-1][0]) > L / 2) | (np.abs(o["state"][-1][1]) > L / 2)
    ph = np.abs(o["phase"]).max()
    dph = np.abs(k["phase"] - o["phase"])
    assert dph[:, ~side].max() <= _tol(precision) * ph
    damp = np.abs(k["amp"].astype(np.float64) - o["amp"])
    assert damp[:, ~side].max() < (1e-12 if precision == "f64" else 1e-6)
    assert (k["steps"] != o["steps"]).mean() < 1e-3


@pytest.mark.parametrize("integ", ["rkn", "rk4"])
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_many_saves_inside_interior_runs(precision, integ):
    """40 saves, every few steps: the tracer's uniform step loop must stop at
    each save inside its interior runs. Against the oracle at every save."""
    n = 48
    h = L / (n - 1)
    ne = workloads.kolmogorov_box(n, L=L, mean=1e25, rms=0.2, seed=41).numpy()
    rays = workloads.gaussian_beam(3000, waist=1.5e-3, L=L, seed=42).numpy()
    sched = runtime.schedule_times(np.linspace(0.0, 1.2 * L, 40), (h, h, h))
    assert sched.n_saves == 40 and sched.save_every >= 2
    kw = dict(inv_brems=True, Te=20.0, Z=1.0, integrator=integ)
    k = run_kernel(ne, rays, (-L / 2,) * 3, (h,) * 3, OMEGA, sched, precision=precision, **kw)
    o = run_oracle(ne, rays, (-L / 2,) * 3, (h,) * 3, OMEGA, sched, **kw)
    assert position_error(k["state"], o["state"], L) < _tol(precision)
    assert direction_error(k["state"], o["state"]) < _tol(precision)
    inside = np.all(np.abs(o["state"][:, :2]) <= L / 2, axis=1)      # (saves, rays) off the side faces
    ph = np.abs(o["phase"]).max()
    assert np.abs(k["phase"] - o["phase"])[inside].max() <= _tol(precision) * ph
    assert (k["steps"] != o["steps"]).mean() < 1e-3
