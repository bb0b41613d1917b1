"""core.propagator for B200: solve / trace_and_save_depths over CUDA kernels.

Mirrors the reference's public functions (src/core/propagator.py):

* ``omega_pe``, ``n_refrac``, ``kappa_inv_brems``     (:31-37, :116-164)
* ``precompute_gradients``                            (:39-93)
* ``dndr``, ``dsdt``                                  (:96-114, :168-243)
* ``solve``                                           (:364-929)
* ``trace_and_save_depths``                           (:932-1234)

with the same signatures, return values and errors (plus keyword-only
extras, below). The ODE is integrated
with a fixed-step fourth-order Runge-Kutta-Nystrom method (step = half the
smallest grid spacing, in c*t) by the sm_100a tracers instead of diffrax's
adaptive Tsit5, so ``jitted``, ``parallelise``, ``rtol`` and ``atol`` are
accepted and have no effect.
Additive keyword-only extras: ``precision`` ('f32' = FP32 kernel with
compensated sums and FP64 phase, 'f64' = all-FP64 kernel), ``detector_plane``
(back-project the final rays to that plane), ``return_extras`` (append a dict
with the optical phase, per-ray status and step counts), ``integrator``
('rkn', the default, or 'rk4': classical RK4 steps, four field samples
instead of three), ``device``, ``stream``,
``group`` (a torch.distributed process group: the job's rays are split over
its ranks, each rank traces its slice through its own copy of the grid, and
every rank returns the results of all rays in their order; see shard.py).
"""
from __future__ import annotations

import pickle
import time
import warnings

import numpy as np
import torch

from .. import runtime, shard
from ..shared.propagation import ray_to_Jonesvector, back_propogate  # noqa: F401  (re-exported as in the reference)
from . import physics
from .beam import Beam

C = physics.C
omega_pe = physics.omega_pe
n_refrac = physics.n_refrac
kappa_inv_brems = physics.kappa_inv_brems


# ---------------------------------------------------------------------------
# Grid helpers
# ---------------------------------------------------------------------------
def _axis_of(probing_direction):
    return ['x', 'y', 'z'].index(probing_direction)


def _geometry(domain):
    o, h, n = zip(*(runtime.uniform_axis(ax) for ax in (domain.x, domain.y, domain.z)))
    return o, h, n


def _scalar(v, name):
    a = np.asarray(v, dtype=np.float64)
    if a.size == 1:
        return float(a.reshape(()))
    if np.all(a == a.flat[0]):
        return float(a.flat[0])
    raise NotImplementedError(f"spatially varying {name} is not supported by the B200 tracers; pass a scalar")


def _check_overcritical(ne, omega, stacklevel=3, ne_max=None):
    ncr = physics.critical_density(omega)
    if ne_max is None:
        ne_max = float(ne.max()) if isinstance(ne, torch.Tensor) else float(np.max(ne))
    if ne_max >= ncr:
        warnings.warn(
            f"precompute_gradients: {ne_max:.3g} m⁻³ cells at or above critical density ncr = {ncr:.3g} m⁻³ "
            f"(ne/ncr = {ne_max/ncr:.2g}).  This causes large gradient magnitudes that prevent ODE convergence.  "
            "Check that ne is in m⁻³ (not cm⁻³ — convert with ne_cc * 1e6) and that your domain does not "
            "include over-critical cells.", stacklevel=stacklevel)


def device_grid(domain, omega, *, precision="f32", device=None, stream=None):
    """Pack the domain's ne into a device grid (K1)."""
    origin, spacing, n = _geometry(domain)
    ne = getattr(domain, "_device_ne", None)
    if ne is None:
        ne = domain.ne
    if isinstance(ne, np.ndarray):
        ne = np.asarray(ne)
    elif not isinstance(ne, torch.Tensor):
        ne = np.asarray(ne)
    if tuple(ne.shape) != tuple(n):
        raise ValueError(f"ne has shape {tuple(ne.shape)} but the coordinates give {tuple(n)}")
    g = runtime.pack_grid(ne, origin, spacing, omega, precision=precision, device=device, stream=stream)
    # the warning uses the maximum the pack's device reduction already found
    _check_overcritical(ne, omega, stacklevel=4, ne_max=g.ne_max)
    return g


def precompute_gradients(ne, x, y, z, omega, *, device=None):
    """Gradients of G = -c^2/2 * ne/nc along x, y, z (propagator.py:39-93),
    computed on the device by K1 (FP64 arithmetic); returns three numpy
    float64 arrays of ne's shape. Warns when ne reaches the critical density."""
    _check_overcritical(ne, omega)
    origin, spacing, _ = zip(*(runtime.uniform_axis(a) for a in (x, y, z)))
    g = runtime.pack_grid(ne if isinstance(ne, torch.Tensor) else np.asarray(ne), origin, spacing, omega,
                          precision="f64", device=device, layout="values")
    n = g.n
    v = g.data.view(*n, 4).cpu().numpy()
    return tuple(-0.5 * C ** 2 * v[..., 1 + a] / spacing[a] for a in range(3))


def dndr(r, dndx, dndy, dndz, x, y, z):
    """(3, N) trilinear interpolation of the three gradient grids at r (N, 3)
    with fill 0 (propagator.py:96-114), through the device sampler (K0)."""
    r = np.asarray(r, dtype=np.float64).reshape(-1, 3)
    origin, spacing, _ = zip(*(runtime.uniform_axis(a) for a in (x, y, z)))
    out = []
    for d in (dndx, dndy, dndz):
        # the gradient grid becomes the q channel of a unit-scale packed grid
        g = runtime.pack_grid(np.asarray(d, dtype=np.float64), origin, spacing, 1.0, precision="f64",
                              ne_scale=1.0, layout="values")
        out.append(runtime.sample(g, r.T)[0].cpu().numpy())
    return np.stack(out)


def dsdt(t, s, parallelise, dndx, dndy, dndz, x, y, z, lengths, dims, kappa=None):
    """Flattened RHS of the ray ODE (propagator.py:168-243) on the device
    sampler: d(x,y,z)/dt = v, dv/dt = grad G(r), dtau/dt = kappa(r)."""
    nstate = 7 if kappa is not None else 6
    s = np.reshape(np.asarray(s, dtype=np.float64), (nstate, -1)) if not parallelise else \
        np.reshape(np.asarray(s, dtype=np.float64), (nstate, 1))
    r = s[:3].T
    sprime = np.zeros_like(s)
    sprime[3:6] = dndr(r, dndx, dndy, dndz, x, y, z)
    sprime[:3] = s[3:6]
    if kappa is not None:
        origin, spacing, _ = zip(*(runtime.uniform_axis(a) for a in (x, y, z)))
        g = runtime.pack_grid(np.asarray(kappa, dtype=np.float64), origin, spacing, 1.0, precision="f64",
                              ne_scale=1.0, layout="values")
        sprime[6] = runtime.sample(g, r.T)[0].cpu().numpy()
    return np.ravel(sprime)


# ---------------------------------------------------------------------------
# Beam resolution (propagator.py:475-509, :1065-1081)
# ---------------------------------------------------------------------------
def _rays_from(beam, domain, batching_message=True):
    assert not isinstance(beam, Beam), (
        "\nThis function does not take in the direct output of the Beam object, pass either Beam.s0 rays, "
        "or the parameters passed to be Beam here as a tuple if batching rays.")
    if isinstance(beam, tuple):
        Np_total = getattr(domain, "Np_total", None)
        assert Np_total is not None, (
            "\nScalarDomain.Np_total must be set when passing beam as a tuple. "
            "Pass Np=<number_of_rays> to ScalarDomain(...).")
        return Beam(Np_total, beam_size=beam[0], divergence=beam[1], ne_extent=beam[2], probing_direction=beam[3],
                    beam_type=beam[4], seeded=beam[5]).s0
    if isinstance(beam, (np.ndarray, torch.Tensor)) or hasattr(beam, "__array__"):
        assert len(beam.shape) == 2, "\nExpected a matrix of pre-created rays."
        return beam
    assert isinstance(beam, tuple), "\nExpect a tuple of Beam properties if you wish to batch rays."


def _ib_params(domain):
    inv_brems = bool(getattr(domain, "inv_brems", False))
    if not inv_brems:
        return False, None, None
    return True, _scalar(domain.Te, "Te"), _scalar(domain.Z, "Z")


class RawSolution:
    """Stand-in for the diffrax Solution the reference returns with
    return_raw_results=True: ys (N, saves, 6 or 7), ts (N, saves) normalised time."""

    def __init__(self, ys, ts):
        self.ys = ys
        self.ts = ts


# ---------------------------------------------------------------------------
# solve (propagator.py:364-929)
# ---------------------------------------------------------------------------
def _traced(grid, rays, sched, *, want, chunk_rays, group, dev, **kw):
    """runtime.trace_to_host over all rays, or, with a process group, over this
    rank's slice followed by the all-gather of every output into ray order
    (total ray-steps summed, time the longest over the ranks)."""
    if group is None:
        return runtime.trace_to_host(grid, rays, sched, want=want, chunk_rays=chunk_rays, **kw)
    world, rank = shard.group_info(group)
    n = int(rays.shape[1])
    lo, hi = shard.shard_bounds(n, world, rank)
    host, total_steps, duration = runtime.trace_to_host(grid, rays[:, lo:hi], sched, want=want,
                                                        chunk_rays=chunk_rays, **kw)
    cdev = shard.comm_device(group, dev)
    host = {k: shard.gather_rays(v, n, group, cdev) for k, v in host.items()}
    return host, int(shard.reduce_scalar(total_steps, group, cdev, "sum")), \
        shard.reduce_scalar(duration, group, cdev, "max")


def solve(beam, ScalarDomain, probing_depth, *, parallelise=True, jitted=True, save_points_per_region=2,
          memory_debug=False, lwl=1064e-9, keep_domain=False, return_raw_results=False, verbose=True,
          precision="f32", detector_plane=None, return_extras=False, device=None, stream=None,
          chunk_rays=None, group=None, integrator="rkn"):
    """Trace rays through the domain to c*t = sqrt(8)*probing_depth (the
    reference's integration end, :616-617) and return (rf, amp, duration).

    rf is the (4, N) Jones vector (x, angle_x, y, angle_y for probing 'z') of
    the rays' current position (keep_current_plane=True, :316-327); with
    save_points_per_region > 2 it is stacked (S, 4, N) over the save times
    linspace(0, 1, S)*sqrt(8)*probing_depth/c and amp is None, as in the
    reference. amp = exp(-tau) when ScalarDomain.inv_brems. duration is the
    wall time of the trace in seconds (numpy float64), including the rays'
    and results' copies, which overlap it.

    The rays pass through the device in chunks of ``chunk_rays`` (default
    ``runtime.STREAM_CHUNK_RAYS``); the results do not depend on it. With a
    process group every rank passes the same beam and domain; each traces
    its slice of the rays and returns the results of all of them.
    """
    omega = physics.omega_of(lwl)
    region_count = getattr(ScalarDomain, "region_count", 1)
    if verbose:
        print("\nNumber of domain batches:", region_count)
        print("Number of ray batches:", getattr(ScalarDomain, "ray_batch_count", 1))
    rays = _rays_from(beam, ScalarDomain)
    dev = runtime.require_device(device)
    axis = _axis_of(ScalarDomain.probing_direction)
    inv_brems, Te, Z = _ib_params(ScalarDomain)
    grid = device_grid(ScalarDomain, omega, precision=precision, device=dev, stream=stream)
    T = np.sqrt(8.0) * float(probing_depth)
    S = int(save_points_per_region)
    taus = np.linspace(0.0, T, S) if S > 1 else np.array([0.0])
    sched = runtime.schedule_times(taus, grid.spacing) if S > 1 else runtime.Schedule(runtime.nominal_step(grid.spacing), 0, 1, 1)
    project = detector_plane is not None
    # rays stream through the device in chunks; their host<->device copies
    # overlap the tracing of the neighbouring chunks
    want = {}
    if return_raw_results:
        want["state"] = "all"
        if inv_brems:
            want["amp"] = "all"
    else:
        want["jones"] = "last" if S <= 2 else "all"
        if S <= 2 and inv_brems:
            want["amp"] = "last"
    if return_extras:
        want.update(phase="all", status="all", steps="all")
    host, total_steps, duration = _traced(
        grid, rays, sched, want=want, chunk_rays=chunk_rays, group=group, dev=dev, axis=axis, project=project,
        plane=float(detector_plane) if project else 0.0, inv_brems=inv_brems, Te=Te, Z=Z, stream=stream,
        integrator=integrator)
    duration = np.float64(duration)
    if verbose:
        print("\nCompleted ray trace in", np.round(duration, 3), "seconds.")
    extras = None
    if return_extras:
        extras = {"phase": host["phase"], "status": host["status"], "steps": host["steps"],
                  "total_steps": total_steps, "precision": precision}

    def ret(*v):
        return (*v, extras) if return_extras else v

    if return_raw_results:
        ys = np.transpose(host["state"], (2, 0, 1))          # (N, S, 6)
        if inv_brems:
            tau = -np.log(host["amp"].astype(np.float64))    # (S, N)
            ys = np.concatenate([ys, tau.T[:, :, None]], axis=2)
        ts = np.broadcast_to(np.linspace(0.0, 1.0, S)[None, :], (ys.shape[0], S))
        return ret(np.asarray([RawSolution(ys, ts)], dtype=object), None, duration)
    if S <= 2:
        return ret(host["jones"], host.get("amp"), duration)
    return ret(host["jones"], None, duration)


# ---------------------------------------------------------------------------
# trace_and_save_depths (propagator.py:932-1234)
# ---------------------------------------------------------------------------
def trace_and_save_depths(beam, ScalarDomain, step, depth_max, output_path, *, lwl=1064e-9, jones_components=None,
                          jitted=True, rtol=1e-3, atol=1e-5, verbose=True, precision="f32", return_extras=False,
                          device=None, stream=None, chunk_rays=None, group=None, integrator="rkn"):
    """Trace rays and save the Jones vector at depths 0, step, ..., depth_max
    (c*t = depth, :1133-1138); returns {'depth_saves', 'jvec',
    'jones_components'[, 'amplitude']} and optionally pickles it. The rays
    pass through the device in chunks of ``chunk_rays``, and split over a
    process group's ranks with ``group``, as in ``solve``."""
    omega = physics.omega_of(lwl)
    s0 = _rays_from(beam, ScalarDomain)
    if step <= 0 or depth_max <= 0:
        raise ValueError("step and depth_max must be positive.")
    if jones_components is None or (isinstance(jones_components, str) and jones_components == 'all'):
        comp = [0, 1, 2, 3]
    elif isinstance(jones_components, str) and jones_components == 'position':
        comp = [0, 2]
    elif isinstance(jones_components, str) and jones_components == 'angle':
        comp = [1, 3]
    else:
        comp = list(jones_components)
        invalid = [i for i in comp if i not in (0, 1, 2, 3)]
        if invalid:
            raise ValueError(f"jones_components indices {invalid} are out of range. Valid indices are 0, 1, 2, 3.")
    probing_direction = ScalarDomain.probing_direction
    axis = _axis_of(probing_direction)
    trace_depth = float(ScalarDomain.lengths[axis])
    if trace_depth < depth_max:
        raise ValueError(
            f"Domain length in probing direction '{probing_direction}' ({trace_depth:.6g} m) "
            f"is smaller than the requested depth_max ({depth_max:.6g} m). "
            f"Increase the domain size to at least depth_max.")
    n_saves = int(np.round(depth_max / step)) + 1
    depth_saves = np.linspace(0.0, depth_max, n_saves)
    inv_brems, Te, Z = _ib_params(ScalarDomain)
    if verbose:
        print(f"\ntrace_and_save_depths: saving at {n_saves} depth(s) from 0 to {depth_max*1e3:.4g} mm "
              f"(step = {step*1e6:.4g} µm, probing direction = '{probing_direction}', "
              f"jones_components = {comp}, inv_brems = {inv_brems}).")
    if n_saves > runtime.capi.SLOTH_MAX_SAVES:
        raise ValueError(f"at most {runtime.capi.SLOTH_MAX_SAVES} depth saves are supported")
    dev = runtime.require_device(device)
    grid = device_grid(ScalarDomain, omega, precision=precision, device=dev, stream=stream)
    sched = runtime.schedule_times(depth_saves, grid.spacing)
    want = {k: "all" for k in ["jones"] + (["amp"] if inv_brems else []) +
            (["phase", "status", "steps"] if return_extras else [])}
    host, _, _ = _traced(grid, s0, sched, want=want, chunk_rays=chunk_rays, group=group, dev=dev, axis=axis,
                         inv_brems=inv_brems, Te=Te, Z=Z, stream=stream, integrator=integrator)
    jones = host["jones"]
    jvec = [np.asarray(jones[j])[comp, :] for j in range(n_saves)]
    result = {'depth_saves': depth_saves, 'jvec': jvec, 'jones_components': comp}
    if inv_brems:
        amp = host["amp"]
        result['amplitude'] = [np.asarray(amp[j]) for j in range(n_saves)]
    if return_extras:
        result['phase'] = [p for p in host["phase"]]
        result['status'] = host["status"]
        result['steps'] = host["steps"]
    if output_path is not None and (group is None or shard.group_info(group)[1] == 0):
        with open(output_path, 'wb') as fh:
            pickle.dump(result, fh)
        if verbose:
            print(f"trace_and_save_depths: results saved to '{output_path}'.")
    return result
