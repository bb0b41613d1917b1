"""The oracle is pinned to the reference: golden vectors from the reference's
own code (tests/golden/make_golden.py) and the analytic trough of the
reference's test module. CPU only."""
import numpy as np
import pytest

from conftest import golden
from oracle import oracle_c
from oracle import ref_restated as rr

C = rr.C


def test_precompute_gradients_golden():
    g = golden("precompute_gradients")
    got = rr.precompute_gradients(g["ne"], g["x"], g["y"], g["z"], float(g["omega"]))
    for k, name in enumerate(("dndx", "dndy", "dndz")):
        np.testing.assert_allclose(got[k], g[name], rtol=1e-14, atol=0)
    got32 = rr.precompute_gradients(g["ne"].astype(np.float32), g["x"].astype(np.float32),
                                    g["y"].astype(np.float32), g["z"].astype(np.float32), float(g["omega"]))
    for k, name in enumerate(("dndx32", "dndy32", "dndz32")):
        np.testing.assert_array_equal(got32[k], g[name])


def test_pack_grid_is_precompute_gradients():
    """The kernel layout (q, dq per cell) carries the same gradients."""
    g = golden("precompute_gradients")
    omega = float(g["omega"])
    nc = rr.critical_density(omega)
    packed = rr.pack_grid(g["ne"], 1.0 / nc)
    for k, (name, ax) in enumerate((("dndx", g["x"]), ("dndy", g["y"]), ("dndz", g["z"]))):
        h = (ax[-1] - ax[0]) / (ax.size - 1)
        np.testing.assert_allclose(-0.5 * C ** 2 * packed[..., 1 + k] / h, g[name], rtol=1e-11)
    np.testing.assert_array_equal(packed[..., 0], g["ne"] * (1.0 / nc))


def test_kappa_golden_and_factorisation():
    cases = golden("kappa")["cases"]
    for ne, Te, Z, om, kref in cases:
        assert rr.kappa_inv_brems(ne, Te, Z, om) == pytest.approx(kref, rel=1e-14)
        kq2, clw, ope2 = rr.kappa_factors(Te, Z, om)
        q = ne / rr.critical_density(om)
        cl = max(2.0, clw - 0.5 * np.log(max(ope2 * q, 1.0)))
        assert kq2 * q * q * cl * C == pytest.approx(kref, rel=1e-12)


def test_interpolator_golden():
    g = golden("interpolator")
    got = rr.regular_grid_interpolator((g["x"], g["y"], g["z"]), g["values"], g["points"])
    np.testing.assert_allclose(got, g["result"], rtol=1e-14, atol=1e-15)
    # the uniform-grid form the kernels use agrees with searchsorted
    grid = rr.Grid(np.zeros(g["values"].shape), (g["x"][0], g["y"][0], g["z"][0]),
                   [(a[-1] - a[0]) / (a.size - 1) for a in (g["x"], g["y"], g["z"])], 1.0)
    grid.fields[..., 1] = g["values"]
    f, _, _ = grid.sample(g["points"].T)
    np.testing.assert_allclose(f[:, 1], g["result"], rtol=1e-12, atol=1e-13)


def test_dsdt_golden():
    g = golden("dsdt")
    pg = golden("precompute_gradients")
    grads = rr.precompute_gradients(pg["ne"], pg["x"], pg["y"], pg["z"], float(pg["omega"]))
    for k in range(g["states"].shape[1]):
        sp = rr.dsdt(0.0, g["states"][:, k], True, *grads, pg["x"], pg["y"], pg["z"], None, None, g["kappa"])
        np.testing.assert_allclose(sp, g["sprime"][:, k], rtol=1e-14, atol=1e-30)


def test_jones_golden():
    g = golden("jones")
    for d in "xyz":
        for keep in (True, False):
            got, _ = rr.ray_to_Jonesvector(g["rays"], ne_extent=1.5e-3, probing_direction=d, keep_current_plane=keep)
            np.testing.assert_allclose(got, g[f"{d}_{int(keep)}"], rtol=1e-15, atol=0)
        np.testing.assert_allclose(rr.back_propogate(g["rays"], 1.5e-3, d), g[f"bp_{d}"], rtol=1e-15, atol=0)


# ---------------------------------------------------------------------------
# Trajectories: the oracle's fixed-step integrator against the reference's own
# trace_and_save_depths / solve run with a tight DOP853 integrator.
# ---------------------------------------------------------------------------
def _trough_grid(ne0, n_xy, n_z, Te=None, Z=None):
    A, HALF_Z = 5e-3, 11e-3
    xs = np.linspace(-A, A, n_xy).astype(np.float32)
    zs = np.linspace(-HALF_Z, HALF_Z, n_z).astype(np.float32)
    XX, _, _ = np.meshgrid(np.linspace(-A, A, n_xy), np.linspace(-A, A, n_xy), np.linspace(-HALF_Z, HALF_Z, n_z),
                           indexing="ij")
    ne = (ne0 * (XX / A) ** 2).astype(np.float32)
    omega = 2 * np.pi * C / 1064e-9
    origin = (float(xs[0]), float(xs[0]), float(zs[0]))
    spacing = ((float(xs[-1]) - float(xs[0])) / (n_xy - 1),) * 2 + ((float(zs[-1]) - float(zs[0])) / (n_z - 1),)
    return rr.Grid(ne, origin, spacing, omega, Te=Te, Z=Z)


def _depth_schedule(grid, depth_saves):
    h = 0.5 * min(grid.spacing)
    d = depth_saves[1] - depth_saves[0]
    m = int(np.ceil(d / h - 1e-9))
    return dict(dtau=d / m, first_save=0, save_every=m, n_saves=len(depth_saves))


def _assert_jones(got, ref, pos_atol, ang_atol):
    """Positions (rows 0, 2) in metres and angles (rows 1, 3) in radians."""
    got, ref = np.asarray(got), np.asarray(ref)
    np.testing.assert_allclose(got[..., [0, 2], :], ref[..., [0, 2], :], rtol=0, atol=pos_atol)
    np.testing.assert_allclose(got[..., [1, 3], :], ref[..., [1, 3], :], rtol=0, atol=ang_atol)


@pytest.mark.parametrize("integ", ["rkn", "rk4"])
def test_trough_matches_reference_and_analytic(integ):
    t = golden("trace_cases")
    grid = _trough_grid(float(t["trough_ne0"]), 24, 24)
    sch = _depth_schedule(grid, t["trough_depths"])
    res = rr.trace_rays(grid, t["trough_s0"].astype(np.float64), integrator=integ, **sch)
    x0 = np.array([0.5e-3, 1.0e-3, 1.5e-3, 2.0e-3])
    # reference (DOP853) vs the fixed-step integrator, and analytic SHM x0*cos(pi/4)
    _assert_jones(res["jones"][-1], t["trough_jvec"][-1], 2e-9, 2e-8)
    np.testing.assert_allclose(res["jones"][-1][0], x0 / np.sqrt(2), rtol=0, atol=2e-9)
    # vx = -x0*Omega*sin(pi/4) within the reference test's 10 %
    omega_osc = (np.pi / 4) / (20e-3 / C)
    np.testing.assert_allclose(res["jones"][-1][1] * C, -x0 * omega_osc * np.sin(np.pi / 4), rtol=0.10)


@pytest.mark.parametrize("integ", ["rkn", "rk4"])
def test_trough_inv_brems_matches_reference(integ):
    t = golden("trace_cases")
    grid = _trough_grid(float(t["trough_ne0"]), 20, 20, Te=100.0, Z=1.0)
    sch = _depth_schedule(grid, t["trough_ib_depths"])
    res = rr.trace_rays(grid, t["trough_s0"].astype(np.float64), inv_brems=True, integrator=integ, **sch)
    _assert_jones(res["jones"], t["trough_ib_jvec"], 5e-9, 2e-8)
    # kappa(r) along a path is only piecewise smooth (trilinear, kinks at cell
    # faces): the fixed-step quadrature differs from tight DOP853 by ~1e-5 here.
    np.testing.assert_allclose(res["amp"], t["trough_ib_amp"], rtol=0, atol=2e-5)


@pytest.mark.parametrize("integ", ["rkn", "rk4"])
def test_uniform_absorption_matches_reference_and_formula(integ):
    t = golden("trace_cases")
    n, half = 16, 3e-3
    coords = np.linspace(-half, half, n).astype(np.float32)
    h = (float(coords[-1]) - float(coords[0])) / (n - 1)
    omega = 2 * np.pi * C / 1064e-9
    grid = rr.Grid(np.full((n, n, n), 1e25, dtype=np.float32), (float(coords[0]),) * 3, (h,) * 3, omega,
                   Te=100.0, Z=1.0)
    sch = _depth_schedule(grid, t["uniform_depths"])
    res = rr.trace_rays(grid, t["uniform_s0"].astype(np.float64), inv_brems=True, integrator=integ, **sch)
    np.testing.assert_allclose(res["amp"], t["uniform_amp"], rtol=0, atol=5e-9)   # float32 kappa grid in the reference
    _assert_jones(res["jones"], t["uniform_jvec"], 1e-9, 5e-9)
    # amp = exp(-kappa*d/c) of the reference test (5 %): exact here up to n < 1
    kappa = rr.kappa_inv_brems(np.float32(1e25), np.float32(100.0), 1.0, omega)
    assert res["amp"][-1].mean() == pytest.approx(np.exp(-kappa * 2e-3 / C), rel=1e-4)


@pytest.mark.parametrize("integ", ["rkn", "rk4"])
def test_solve_end_state_matches_reference(integ):
    """solve() integrates to c*t = sqrt(8)*depth and reports the current plane."""
    t = golden("trace_cases")
    grid = _trough_grid(float(t["trough_ne0"]), 24, 24)
    T = np.sqrt(8.0) * float(t["solve_depth"])
    h = 0.5 * min(grid.spacing)
    m = int(np.ceil(T / h - 1e-9))
    res = rr.trace_rays(grid, t["trough_s0"].astype(np.float64), dtau=T / m, first_save=m, save_every=1,
                        n_saves=1, integrator=integ)
    _assert_jones(res["jones"][-1], t["solve_rf"], 5e-9, 2e-8)


# ---------------------------------------------------------------------------
# Oracle self-consistency: C vs numpy, early exit vs plain stepping.
# ---------------------------------------------------------------------------
def _sinus_case(n=24, nrays=200, seed=3, axis=2, Te=None):
    rng = np.random.RandomState(seed)
    L = 5e-3
    c1 = np.linspace(-L / 2, L / 2, n)
    X, Y, Z = np.meshgrid(c1, c1, c1, indexing="ij")
    ne = 1e25 * (1 + 0.1 * np.sin(2 * np.pi * X / 0.5e-3) + 0.05 * np.cos(2 * np.pi * Y / 0.7e-3)
                 + 0.03 * np.sin(2 * np.pi * Z / 0.9e-3))
    omega = 2 * np.pi * C / 532e-9
    grid = rr.Grid(ne, (-L / 2,) * 3, (L / (n - 1),) * 3, omega, Te=Te, Z=None if Te is None else 1.0)
    rays = np.zeros((6, nrays))
    t1, t2 = [a for a in range(3) if a != axis]
    rays[t1] = rng.normal(0, 1e-3, nrays)
    rays[t2] = rng.normal(0, 1e-3, nrays)
    rays[axis] = -L / 2
    ang = rng.normal(0, 5e-3, (2, nrays))
    rays[3 + t1] = C * np.sin(ang[0])
    rays[3 + t2] = C * np.sin(ang[1])
    rays[3 + axis] = C * np.sqrt(1 - np.sin(ang[0]) ** 2 - np.sin(ang[1]) ** 2)
    return grid, rays


@pytest.mark.parametrize("axis,project,ib,integ", [(2, False, False, "rkn"), (0, True, True, "rkn"),
                                                   (1, False, True, "rkn"), (2, True, True, "rk4"),
                                                   (0, False, False, "rk4")])
def test_c_oracle_matches_numpy_oracle(axis, project, ib, integ):
    grid, rays = _sinus_case(axis=axis, Te=20.0 if ib else None)
    h = 0.5 * min(grid.spacing)
    kw = dict(dtau=h, first_save=0, save_every=60, n_saves=5, axis=axis, project=project, plane=2.5e-3,
              inv_brems=ib, integrator=integ)
    a = rr.trace_rays(grid, rays, **kw)
    b = oracle_c.trace_rays(grid, rays, **kw)
    np.testing.assert_allclose(b["state"], a["state"], rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(b["jones"], a["jones"], rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(b["phase"], a["phase"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(b["tau"], a["tau"], rtol=1e-12, atol=1e-15)
    np.testing.assert_array_equal(b["steps"], a["steps"])
    np.testing.assert_array_equal(b["status"], a["status"])


def test_early_exit_is_exact_drift():
    grid, rays = _sinus_case(nrays=100, Te=20.0)
    h = 0.5 * min(grid.spacing)
    kw = dict(dtau=h, first_save=0, save_every=40, n_saves=8, inv_brems=True)
    a = oracle_c.trace_rays(grid, rays, early_exit=True, **kw)
    b = oracle_c.trace_rays(grid, rays, early_exit=False, **kw)
    np.testing.assert_allclose(a["state"], b["state"], rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(a["phase"], b["phase"], rtol=1e-13, atol=1e-13)
    assert (a["steps"] <= b["steps"]).all() and a["steps"].sum() < b["steps"].sum()


def test_vacuum_rays_are_straight():
    n = 16
    grid = rr.Grid(np.zeros((n, n, n)), (-2e-3,) * 3, (4e-3 / (n - 1),) * 3, 2 * np.pi * C / 1064e-9)
    rays = np.zeros((6, 2))
    rays[0] = [0.5e-3, 1.0e-3]
    rays[2] = -2e-3
    rays[5] = C
    res = oracle_c.trace_rays(grid, rays, dtau=4e-3 / 60, first_save=60, save_every=1, n_saves=1)
    np.testing.assert_allclose(res["jones"][0][0], rays[0], atol=1e-15)
    assert (res["phase"] == 0).all()


PHASE_CASES = ("smooth_532", "dense_1064", "holes_532")


@pytest.mark.parametrize("name", PHASE_CASES)
def test_reference_phase_integrand_golden(name):
    """The oracle's reference-semantics phase integrand, omega * (interp(n - 1)),
    equals the legacy solver's own ScalarDomain.phase (src/legacy/full_solver.py:342-345,
    interp(n) - 1 with fill n = 1) at inside, outside, node and face points."""
    g = golden("phase")
    ne, pts, ref = g[f"{name}_ne"], g[f"{name}_points"], g[f"{name}_phase"]
    ax = [g[f"{name}_{a}"] for a in "xyz"]
    grid = rr.Grid(ne, [a[0] for a in ax], [a[1] - a[0] for a in ax], float(g[f"{name}_omega"]))
    _, _, nm1 = grid.sample(pts, with_nm1=True)
    got = grid.omega * nm1
    scale = np.abs(ref).max()
    assert np.abs(got - ref).max() <= 1e-12 * scale
    outside = np.zeros(pts.shape[1], dtype=bool)
    for a in range(3):
        outside |= (pts[a] < ax[a][0]) | (pts[a] > ax[a][-1])
    assert outside.sum() > 10 and np.all(ref[outside] == 0.0)


@pytest.mark.parametrize("name", PHASE_CASES)
def test_trace_layout_phase_channel_golden(name):
    """The tracers interpolate channel 0 of the trace layout, n - 1 at the grid
    points (rr.pack_grid with ope_ratio2, the K1 formula): times omega it is
    the legacy solver's ScalarDomain.phase at every golden point."""
    g = golden("phase")
    ne, pts, ref = g[f"{name}_ne"], g[f"{name}_points"], g[f"{name}_phase"]
    ax = [g[f"{name}_{a}"] for a in "xyz"]
    omega = float(g[f"{name}_omega"])
    packed = rr.pack_grid(ne, 1.0 / rr.critical_density(omega), rr.ope_ratio2(omega))
    got = omega * rr.regular_grid_interpolator(tuple(ax), packed[..., 0], pts.T)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("name", PHASE_CASES)
def test_density_phase_integrand_equals_reference_at_nodes(name):
    """The other semantics, n from the interpolated density (the oracle's
    phase_mode 'density'), agrees with the legacy solver at grid nodes and
    differs between them by the curvature of n(ne) over one cell."""
    g = golden("phase")
    ne, pts, ref = g[f"{name}_ne"], g[f"{name}_points"], g[f"{name}_phase"]
    ax = [g[f"{name}_{a}"] for a in "xyz"]
    omega = float(g[f"{name}_omega"])
    grid = rr.Grid(ne, [a[0] for a in ax], [a[1] - a[0] for a in ax], omega)
    f, _, _ = grid.sample(pts)
    kern = rr.phase_integrand(f[:, 0], omega, grid.nc)
    nodes = slice(400, 412)
    np.testing.assert_allclose(kern[nodes], ref[nodes], rtol=1e-12)
    gap = np.abs(kern - ref).max() / np.abs(ref).max()
    assert gap < (0.2 if name == "dense_1064" else 2e-2)


def test_rk4_and_rkn_agree():
    """Both integrators are fourth order in position and direction; on the
    sinusoid case (h/2 steps) they agree to rounding, and each matches the
    reference's DOP853 trajectories (the tests above)."""
    grid, rays = _sinus_case(nrays=60, Te=20.0)
    L = 5e-3
    h = 0.5 * min(grid.spacing)
    m = int(np.ceil(L / h))
    kw = dict(dtau=L / m, first_save=m, save_every=1, n_saves=1, inv_brems=True)
    a = oracle_c.trace_rays(grid, rays, integrator="rkn", **kw)
    b = oracle_c.trace_rays(grid, rays, integrator="rk4", **kw)
    assert np.array_equal(a["status"], b["status"])
    assert np.abs(a["state"][-1][:3] - b["state"][-1][:3]).max() / L < 1e-12
    assert np.abs(a["tau"] - b["tau"]).max() < 1e-9
