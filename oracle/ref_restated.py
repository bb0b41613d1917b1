"""FP64 CPU restatement of SLOTH's ray-propagation hot path.

TEST INFRASTRUCTURE ONLY. This module is the oracle that the CUDA kernels are
checked against. It may be imported only by ``tests/``, by
``__graft_entry__.smoke()`` and by the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py``; the product package never imports it.

Every function restates the reference (paths relative to the SLOTH repo):

* ``omega_pe``, ``n_refrac``             src/core/propagator.py:31-37
* ``precompute_gradients``               src/core/propagator.py:39-93
* ``kappa_inv_brems``                    src/core/propagator.py:116-164
* ``regular_grid_interpolator``          src/core/interpolator.py:15-105
* ``dndr``, ``dsdt``                     src/core/propagator.py:96-114, :168-243
* ``ray_to_Jonesvector``, ``back_propogate``  src/shared/propagation.py:4-134
* phase integrand omega*(n - 1)          src/legacy/full_solver.py:271-274, :341-347
* ``trace_rays``: the fixed-step fourth-order Runge-Kutta-Nystrom
  integration of dsdt (+ phase) that
  replaces diffrax's adaptive Tsit5 (src/core/propagator.py:731-793) in this
  build, with the reference's time normalisation and save semantics
  (:616-617, :1133-1138) and keep_current_plane projection (:316-327).

Parity is pinned by golden vectors produced by running the reference's own
functions (numpy standing in for jax.numpy, scipy DOP853 standing in for
diffrax) -- see tests/golden/make_golden.py -- and by the analytic trough
cases of tests/test_quadratic_trough.py.
"""
from __future__ import annotations

from itertools import product

import numpy as np
from scipy.constants import c as C
from scipy.constants import e as E_CHARGE
from scipy.constants import epsilon_0 as EPS0

ALPHA = 3.14207787e-4   # m_e * eps0 / e^2, the reference's constant (propagator.py:73, :88)
FACE_MARGIN = 0.02      # cells: steps ending this close to a face sample the inside limit


# ---------------------------------------------------------------------------
# Physics helpers
# ---------------------------------------------------------------------------
def omega_pe(ne_cc):
    """Electron plasma frequency (rad/s) from ne in cm^-3 (propagator.py:31-33)."""
    return 5.64e4 * np.sqrt(ne_cc)


def n_refrac(ne, omega):
    """Plasma refractive index from ne in m^-3 (propagator.py:36-37)."""
    return np.sqrt(1.0 - (omega_pe(ne * 1e-6) / omega) ** 2)


def ope_ratio2(omega):
    """(omega_pe/omega)^2 per unit ne/nc with the NRL omega_pe (5.64e4 rad/s per
    sqrt(cm^-3), full_solver.py:236-239) and nc = ALPHA omega^2."""
    return float((5.64e4 ** 2) * critical_density(omega) * 1e-6 / float(omega) ** 2)


def critical_density(omega):
    """ncr = m_e eps0 omega^2 / e^2 in m^-3 (propagator.py:73)."""
    return ALPHA * float(omega) ** 2


def precompute_gradients(ne, x, y, z, omega):
    """Gradient of the driving term G = -c^2/2 * ne/nc (propagator.py:39-93).

    The coefficient is formed in float64 and cast to ne's dtype (:88-89); the
    gradient uses the coordinate arrays, second-order inside and first-order
    one-sided at the faces (jnp.gradient semantics, :90-92).
    """
    ne = np.asarray(ne)
    coeff = np.float64(-0.5) * float(C) ** 2 / (ALPHA * float(omega) ** 2)
    g = ne * ne.dtype.type(coeff)
    return (np.gradient(g, np.asarray(x), axis=0),
            np.gradient(g, np.asarray(y), axis=1),
            np.gradient(g, np.asarray(z), axis=2))


def kappa_inv_brems(ne, Te, Z, omega):
    """Inverse-bremsstrahlung amplitude absorption rate in 1/s (propagator.py:116-164)."""
    ne_cc = np.asarray(ne) * 1e-6
    v_the = 4.19e5 * np.sqrt(Te)
    o_pe = 5.64e4 * np.sqrt(ne_cc)
    o_max = np.maximum(o_pe, omega)
    b_min = Z * E_CHARGE / (4.0 * np.pi * EPS0 * Te)
    CL = np.maximum(2.0, np.log(v_the / (o_max * b_min)))
    return 3.1e-5 * Z * C * (ne_cc / omega) ** 2 * CL * Te ** (-1.5)


def kappa_factors(Te, Z, omega):
    """The tracer's factorisation of kappa for uniform Te, Z: kappa/c =
    kappa_q2 * q^2 * CL(q) with q = ne/nc and CL(q) = max(2, cl_w -
    0.5*ln(max(ope2*q, 1))), ope2 = (omega_pe/omega)^2 per unit q."""
    nc = critical_density(omega)
    kappa_q2 = 3.1e-5 * Z * (nc * 1e-6 / omega) ** 2 * Te ** (-1.5)
    v_the = 4.19e5 * np.sqrt(Te)
    b_min = Z * E_CHARGE / (4.0 * np.pi * EPS0 * Te)
    cl_w = np.log(v_the / (omega * b_min))
    ope2 = (5.64e4 ** 2) * nc * 1e-6 / omega ** 2
    return float(kappa_q2), float(cl_w), float(ope2)


# ---------------------------------------------------------------------------
# Kernel-layout grid (what K1 writes)
# ---------------------------------------------------------------------------
def n_minus_1(x):
    """n - 1 = sqrt(1 - x) - 1 of x = (omega_pe/omega)^2 as -x / (1 + sqrt(1 - x))
    (no cancellation; equal to the legacy n_refrac - 1, full_solver.py:292-296,
    to rounding), and -x above the critical density where the legacy n is
    not real. Every operation is one IEEE rounding, as in the K1 kernel."""
    x = np.asarray(x, dtype=np.float64)
    return -(x / (1.0 + np.sqrt(np.maximum(1.0 - x, 0.0))))


def pack_grid(ne, ne_scale, ope_ratio2=None):
    """(nx, ny, nz, 4) float64: channel 0 and dq per grid cell along each axis,
    central inside and one-sided at the faces, with q = ne*ne_scale; the same
    formula as the K1 kernel, in the same operation order. Channel 0 is q
    (the value layout) or, given ope_ratio2, n - 1 of x = ope_ratio2 * q
    (the trace layout)."""
    q = np.asarray(ne, dtype=np.float64) * ne_scale
    out = np.empty(q.shape + (4,), dtype=np.float64)
    out[..., 0] = q if ope_ratio2 is None else n_minus_1(ope_ratio2 * q)
    for ax in range(3):
        d = np.empty_like(q)
        sl = [slice(None)] * 3

        def s(a, b):
            t = list(sl)
            t[ax] = slice(a, b)
            return tuple(t)
        d[s(1, -1)] = 0.5 * (q[s(2, None)] - q[s(None, -2)])
        d[s(0, 1)] = q[s(1, 2)] - q[s(0, 1)]
        d[s(-1, None)] = q[s(-1, None)] - q[s(-2, -1)]
        out[..., 1 + ax] = d
    return out


# ---------------------------------------------------------------------------
# Interpolation and RHS
# ---------------------------------------------------------------------------
def regular_grid_interpolator(points, values, xi, fill_value=0.0):
    """Trilinear interpolation on a rectilinear grid (interpolator.py:79-104):
    i = searchsorted(g, x) - 1 clamped to [0, n-2], t = (x - g_i)/(g_{i+1} - g_i),
    sum over the 8 corners of value * prod(weights), fill outside."""
    grid = tuple(np.asarray(p, dtype=np.float64) for p in points)
    values = np.asarray(values)
    xi = np.asarray(xi, dtype=np.float64).reshape(-1, len(grid))
    indices, dist = [], []
    oob = np.zeros(xi.shape[0], dtype=bool)
    for x, g in zip(xi.T, grid):
        i = np.searchsorted(g, x) - 1
        i = np.where(i < 0, 0, i)
        i = np.where(i > g.size - 2, g.size - 2, i)
        indices.append(i)
        dist.append((x - g[i]) / (g[i + 1] - g[i]))
        oob |= x < g[0]
        oob |= x > g[-1]
    result = np.zeros(xi.shape[0], dtype=np.float64)
    for edge in product(*[[i, i + 1] for i in indices]):
        w = np.ones(xi.shape[0], dtype=np.float64)
        for ei, i, t in zip(edge, indices, dist):
            w = w * np.where(ei == i, 1 - t, t)
        result = result + values[edge] * w
    if fill_value is not None:
        result = np.where(oob, fill_value, result)
    return result


def dndr(r, dndx, dndy, dndz, x, y, z):
    """(3, N) interpolated gradient of the driving term (propagator.py:96-114)."""
    pts = (x, y, z)
    return np.stack([regular_grid_interpolator(pts, d, r) for d in (dndx, dndy, dndz)])


def dsdt(t, s, parallelise, dndx, dndy, dndz, x, y, z, lengths, dims, kappa=None):
    """Flattened RHS of the ray ODE (propagator.py:168-243)."""
    nstate = 7 if kappa is not None else 6
    s = np.reshape(s, (nstate, -1)) if not parallelise else np.reshape(s, (nstate, 1))
    sprime = np.zeros_like(s, dtype=np.float64)
    r = s[:3, :].T
    sprime[3:6, :] = dndr(r, dndx, dndy, dndz, x, y, z)
    sprime[:3, :] = s[3:6, :]
    if kappa is not None:
        sprime[6, :] = regular_grid_interpolator((x, y, z), kappa, r, fill_value=0.0)
    return np.ravel(sprime)


# ---------------------------------------------------------------------------
# Projection
# ---------------------------------------------------------------------------
def ray_to_Jonesvector(rays, *, ne_extent=None, probing_direction='z', keep_current_plane=False):
    """(4, N) rows (pos1, angle1, pos2, angle2) (propagation.py:4-90)."""
    if ne_extent is None and not keep_current_plane:
        keep_current_plane = True
    x, y, z, vx, vy, vz = [np.asarray(rays[k], dtype=np.float64) for k in range(6)]
    out = np.zeros((4, x.shape[0]))
    if probing_direction == 'x':
        a, t1, t2, va, v1, v2 = x, y, z, vx, vy, vz
    elif probing_direction == 'y':
        a, t1, t2, va, v1, v2 = y, x, z, vy, vx, vz
    elif probing_direction == 'z':
        a, t1, t2, va, v1, v2 = z, x, y, vz, vx, vy
    else:
        return out, None
    if keep_current_plane:
        out[0], out[2] = t1, t2
    else:
        t_bp = (a - ne_extent) / va
        out[0], out[2] = t1 - v1 * t_bp, t2 - v2 * t_bp
    out[1] = np.arctan(v1 / va)
    out[3] = np.arctan(v2 / va)
    return out, None


def back_propogate(rays, ne_extent, probing_direction):
    """Move rays along v onto the plane probing_axis = ne_extent (propagation.py:92-134)."""
    rays = np.array(rays, dtype=np.float64, copy=True)
    ax = {'x': 0, 'y': 1, 'z': 2}[probing_direction]
    t_bp = (rays[ax] - ne_extent) / rays[3 + ax]
    for k in range(3):
        rays[k] = ne_extent if k == ax else rays[k] - rays[3 + k] * t_bp
    return rays


# ---------------------------------------------------------------------------
# Fixed-step Runge-Kutta-Nystrom trace (vectorised over rays)
# ---------------------------------------------------------------------------
class Grid:
    """Uniform grid with the fields the trace reads, in SI units: ne (m^-3),
    the three gradient grids of G (m/s^2) and optionally kappa (1/s) and
    n - 1 (reference-semantics phase)."""

    def __init__(self, ne, origin, spacing, omega, Te=None, Z=None):
        self.ne = np.asarray(ne, dtype=np.float64)
        self.n = self.ne.shape
        self.origin = np.asarray(origin, dtype=np.float64)
        self.spacing = np.asarray(spacing, dtype=np.float64)
        self.omega = float(omega)
        self.nc = critical_density(omega)
        coords = [self.origin[a] + self.spacing[a] * np.arange(self.n[a]) for a in range(3)]
        self.coords = coords
        grads = precompute_gradients(self.ne, *coords, omega)
        self.fields = np.stack([self.ne, *grads], axis=-1)       # (nx,ny,nz,4)
        self.kappa = None if Te is None else kappa_inv_brems(self.ne, Te, Z, omega)
        self.nm1 = n_minus_1((omega_pe(self.ne * 1e-6) / self.omega) ** 2)

    def sample(self, r, *, with_kappa=False, with_nm1=False, clip=None):
        """Interpolate the four fields (and kappa / n-1) at r (3, N); 0 outside.
        Points where `clip` (bool (N,)) is set are first clamped into the grid
        in cell units: a clamp in metres can map back to a cell coordinate just
        above n - 1 by rounding, and then sample the fill value instead of the
        field's limit from inside."""
        u = [(r[a] - self.origin[a]) / self.spacing[a] for a in range(3)]
        if clip is not None:
            u = [np.where(clip, np.clip(u[a], 0.0, self.n[a] - 1), u[a]) for a in range(3)]
        oob = np.zeros(r.shape[1], dtype=bool)
        idx, t = [], []
        for a in range(3):
            oob |= ~((u[a] >= 0) & (u[a] <= self.n[a] - 1))
            i = np.clip(np.floor(np.nan_to_num(u[a])), 0, self.n[a] - 2).astype(np.int64)
            idx.append(i)
            t.append(u[a] - i)
        f = np.zeros((r.shape[1], 4))
        k = np.zeros(r.shape[1]) if with_kappa else None
        m = np.zeros(r.shape[1]) if with_nm1 else None
        for e in product((0, 1), repeat=3):
            w = np.ones(r.shape[1])
            for a in range(3):
                w = w * (t[a] if e[a] else 1 - t[a])
            ii = (idx[0] + e[0], idx[1] + e[1], idx[2] + e[2])
            f += self.fields[ii] * w[:, None]
            if with_kappa:
                k += self.kappa[ii] * w
            if with_nm1:
                m += self.nm1[ii] * w
        f[oob] = 0.0
        if with_kappa:
            k[oob] = 0.0
        if with_nm1:
            m[oob] = 0.0
        return f, k, m


def phase_integrand(ne_interp, omega, nc):
    """omega*(n - 1), n = sqrt(1 - (omega_pe/omega)^2) with the NRL omega_pe
    of full_solver.py:236-239, written as -x/(1 + sqrt(1 - x))."""
    ope2 = (5.64e4 ** 2) * 1e-6 / omega ** 2
    x = ope2 * ne_interp
    return -omega * x / (1.0 + np.sqrt(np.maximum(1.0 - x, 0.0)))


def trace_rays(grid: Grid, rays, *, dtau, first_save, save_every, n_saves, axis=2,
               project=False, plane=0.0, inv_brems=False, early_exit=True,
               phase_mode="reference", integrator="rkn"):
    """Fixed-step fourth-order Runge-Kutta-Nystrom integration of dsdt
    (+ phase, + optical depth) in SI units: three samples per step,
    r2 = r + h/2 v + h^2/8 a1, r3 = r + h v + h^2/2 a2, r' = r + h v +
    h^2/6 (a1 + 2 a2), v' = v + h/6 (a1 + 4 a2 + a3), Simpson's weights for
    the phase and the depth.

    Step dt = dtau/c. Save j after step first_save + j*save_every. The RHS is
    discontinuous at the grid faces (gradients inside, fill 0 outside), so a
    step of a ray inside the grid whose straight-line prediction r + v*dt
    leaves the grid is shortened to end on the face (a step of dt*phi,
    phi = the smallest positive (face - r)/(v*dt)); the ray is then frozen and
    advanced to later saves by straight-line drift from its exit time. A ray
    outside the grid on an axis and moving away on it is frozen likewise.
    The last stage point of such a clipped step lies on the face up to
    O(h^2 * acceleration), where the RHS jumps, so the clipped step, and any
    step whose prediction ends within FACE_MARGIN cells of a face, samples its
    stage points clamped into the grid box: it integrates the field's limit
    from inside, as an event-locating adaptive solver does. kappa is the reference's interpolated kappa
    grid; phase_mode 'reference' (the tracers' semantics) interpolates the
    (n - 1) grid as the legacy solver interpolates n (full_solver.py:289),
    'density' takes n from the interpolated density instead.
    integrator 'rk4' takes classical RK4 steps of the first-order system
    instead (four samples, RK4's weights (1, 2, 2, 1)/6 for the integrals).
    Returns a dict of arrays.
    """
    rays = np.asarray(rays, dtype=np.float64)
    N = rays.shape[1]
    dt = dtau / C
    r = rays[:3].copy()
    v = rays[3:6].copy()
    phase = np.zeros(N)
    tau = np.zeros(N)
    steps = np.zeros(N, dtype=np.int64)
    alive = np.ones(N, dtype=bool)
    every = save_every if n_saves > 1 else 0
    last = first_save + (n_saves - 1) * every
    save_steps = [first_save + j * every for j in range(n_saves)]
    out_state = np.zeros((n_saves, 6, N))
    out_phase = np.zeros((n_saves, N))
    out_tau = np.zeros((n_saves, N))
    lo = grid.origin
    hi = grid.origin + grid.spacing * (np.asarray(grid.n) - 1)

    def rhs(rr, clip=None):
        f, k, m = grid.sample(rr, with_kappa=inv_brems, with_nm1=(phase_mode == "reference"),
                              clip=clip if clip is not None and clip.any() else None)
        a = f[:, 1:].T
        if phase_mode == "reference":
            g = grid.omega * m
        else:
            g = phase_integrand(f[:, 0], grid.omega, grid.nc)
        return a, g, (k if inv_brems else np.zeros(rr.shape[1]))

    def inside(rr):
        res = np.ones(rr.shape[1], dtype=bool)
        for a in range(3):
            res &= (rr[a] >= lo[a]) & (rr[a] <= hi[a])
        return res

    def gone(rr, vv):
        res = np.zeros(rr.shape[1], dtype=bool)
        for a in range(3):
            res |= (rr[a] < lo[a]) & (vv[a] <= 0)
            res |= (rr[a] > hi[a]) & (vv[a] >= 0)
        return res

    frozen_t = np.full(N, -1.0)          # time (in steps) at which the ray froze
    j_next = 0

    def record(j, sel, drift_steps):
        ds = np.asarray(drift_steps, dtype=np.float64)
        out_state[j, :3, sel] = (r[:, sel] + v[:, sel] * (ds * dt)).T
        out_state[j, 3:, sel] = v[:, sel].T
        out_phase[j, sel] = phase[sel]
        out_tau[j, sel] = tau[sel]

    step = 0
    while True:
        while j_next < n_saves and save_steps[j_next] == step:
            record(j_next, alive.copy(), 0.0)
            fz = ~alive
            if fz.any():
                record(j_next, fz, step - frozen_t[fz])
            j_next += 1
        if j_next >= n_saves:
            break
        newly = alive & gone(r, v)
        frozen_t[newly] = step
        alive &= ~newly
        idx = np.nonzero(alive)[0]
        if idx.size:
            rr, vv = r[:, idx], v[:, idx]
            # shorten the step of rays that would leave the grid within it
            phi = np.ones(idx.size)
            near = np.zeros(idx.size, dtype=bool)
            ins = inside(rr)
            for a in range(3):
                pn = rr[a] + vv[a] * dt
                marg = FACE_MARGIN * grid.spacing[a]
                near |= ins & ((pn > hi[a] - marg) | (pn < lo[a] + marg))
                with np.errstate(divide="ignore", invalid="ignore"):
                    up = ins & (pn > hi[a])
                    phi = np.where(up, np.minimum(phi, (hi[a] - rr[a]) / (vv[a] * dt)), phi)
                    dn = ins & (pn < lo[a])
                    phi = np.where(dn, np.minimum(phi, (lo[a] - rr[a]) / (vv[a] * dt)), phi)
            split = phi < 1.0
            clamp = split | near
            phi = np.maximum(phi, 0.0)
            h = dt * phi
            # Nystrom's fourth-order Runge-Kutta-Nystrom step (r'' = a(r);
            # three samples), Simpson's weights for the phase and the depth
            a1, g1, k1 = rhs(rr, clamp)
            if integrator == "rk4":
                r2, v2 = rr + 0.5 * h * vv, vv + 0.5 * h * a1
                a2, g2, k2 = rhs(r2, clamp)
                r3, v3 = rr + 0.5 * h * v2, vv + 0.5 * h * a2
                a3, g3, k3 = rhs(r3, clamp)
                r4, v4 = rr + h * v3, vv + h * a3
                a4, g4, k4 = rhs(r4, clamp)
                r[:, idx] = rr + h / 6.0 * (vv + 2 * v2 + 2 * v3 + v4)
                v[:, idx] = vv + h / 6.0 * (a1 + 2 * a2 + 2 * a3 + a4)
                phase[idx] += h / 6.0 * (g1 + 2 * g2 + 2 * g3 + g4)
                tau[idx] += h / 6.0 * (k1 + 2 * k2 + 2 * k3 + k4)
            else:
                r2 = rr + 0.5 * h * vv + (h * h / 8.0) * a1
                a2, g2, k2 = rhs(r2, clamp)
                r3 = rr + h * vv + (h * h / 2.0) * a2
                a3, g3, k3 = rhs(r3, clamp)
                r[:, idx] = rr + h * vv + (h * h / 6.0) * (a1 + 2 * a2)
                v[:, idx] = vv + h / 6.0 * (a1 + 4 * a2 + a3)
                phase[idx] += h / 6.0 * (g1 + 4 * g2 + g3)
                tau[idx] += h / 6.0 * (k1 + 4 * k2 + k3)
            steps[idx] += 1
            if split.any():
                sidx = idx[split]
                frozen_t[sidx] = step + phi[split]
                alive[sidx] = False
        step += 1
        if step > last:
            break
    status = np.where(alive & inside(r), 1, 0).astype(np.uint8)
    status[~np.isfinite(r).all(axis=0) | ~np.isfinite(v).all(axis=0)] = 2
    dirname = "xyz"[axis]
    jones = np.stack([ray_to_Jonesvector(out_state[j], ne_extent=plane, probing_direction=dirname,
                                         keep_current_plane=not project)[0] for j in range(n_saves)])
    return dict(state=out_state, jones=jones, phase=out_phase, tau=out_tau,
                amp=np.exp(-out_tau), steps=steps, status=status)
