"""Parity of the CUDA kernels (through the C ABI) with the oracle on seeded inputs.

Tolerances (stated for every output):
* FP64 kernel vs FP64 oracle: positions 1e-10 of the box length, directions
  1e-10 (|d(v/c)|), phase 1e-10 relative, amplitude 1e-12 absolute.
* FP32 split kernel vs FP64 oracle: positions 1e-6 of the box length and
  directions 1e-6 for every ray; phase 1e-6 relative (of max |phase|) and
  amplitude 1e-6 absolute for rays that leave through the far face or stay
  inside. Rays that leave through a side face do so at grazing incidence
  (normal velocity ~1e-3 c): their exit time, and so the phase and optical
  depth gathered up to it, moves by (position rounding)/(normal velocity);
  for them the bounds are 1e-3 relative and 1e-4 absolute.
"""
import numpy as np
import pytest
import torch

from conftest import golden
from helpers import C, case, direction_error, position_error, run_kernel, run_oracle
from oracle import ref_restated as rr
from sloth_b200 import _capi, runtime, workloads
from sloth_b200.core import physics

pytestmark = pytest.mark.gpu

L = 5e-3


@pytest.mark.parametrize("layout", ["trace", "values"])
@pytest.mark.parametrize("ne_dtype", [np.float32, np.float64])
def test_pack_matches_oracle_bitwise(ne_dtype, layout):
    """Both layouts of K1, bitwise the oracle's FP64 formula (the trace
    layout's n - 1 includes densities above the critical one, where it is -x)."""
    rng = np.random.RandomState(5)
    ne = rng.uniform(1e24, 3e25, size=(9, 10, 11)).astype(ne_dtype)
    omega = 2 * np.pi * C / 532e-9
    nc = rr.critical_density(omega)
    ne[0, 0, :3] = np.array([0.5, 0.999, 2.0]) * nc
    scale = 1.0 / nc
    ope2 = physics.ope_ratio2(omega) if layout == "trace" else None
    ref = rr.pack_grid(ne.astype(np.float64), scale, ope2)
    g64 = runtime.pack_grid(torch.from_numpy(ne), (0, 0, 0), (1e-5,) * 3, omega, precision="f64", layout=layout)
    np.testing.assert_array_equal(g64.data.view(9, 10, 11, 4).cpu().numpy(), ref)
    g32 = runtime.pack_grid(torch.from_numpy(ne), (0, 0, 0), (1e-5,) * 3, omega, precision="f32", layout=layout)
    np.testing.assert_array_equal(g32.data.view(9, 10, 11, 4).cpu().numpy(), ref.astype(np.float32))


@pytest.mark.parametrize("precision,rtol", [("f64", 1e-13), ("f32", 2e-6)])
def test_sample_matches_reference_interpolator(precision, rtol):
    g = golden("interpolator")
    x, y, z = g["x"], g["y"], g["z"]
    origin = (x[0], y[0], z[0])
    spacing = tuple((a[-1] - a[0]) / (a.size - 1) for a in (x, y, z))
    grid = runtime.pack_grid(torch.from_numpy(g["values"]), origin, spacing, 1.0, precision=precision, ne_scale=1.0,
                             layout="values")
    got = runtime.sample(grid, g["points"].T)[0].cpu().numpy().astype(np.float64)
    scale = np.abs(g["values"]).max()
    np.testing.assert_allclose(got, g["result"], rtol=0, atol=rtol * scale)
    out = (g["points"][:, 0] < x[0]) | (g["points"][:, 0] > x[-1])
    assert (got[out] == 0).all()


CASES = [
    # kind, n, nrays, axis, inv_brems, project, n_saves, jitter
    ("sinusoid", 64, 3000, 2, False, False, 1, 0.0),
    ("trough", 48, 2000, 2, True, True, 1, 1e-3),
    ("kolmogorov", 40, 2000, 2, True, False, 4, 0.0),
    ("kolmogorov", 32, 1500, 0, False, True, 1, 2e-3),
    ("sinusoid", 32, 1500, 1, True, False, 3, 5e-3),
]


def _sched(n, n_saves, solve_like):
    h = L / (n - 1)
    if solve_like:
        taus = np.array([np.sqrt(8.0) * L])
    else:
        taus = np.linspace(0.0, L, n_saves)
    return runtime.schedule_times(taus, (h, h, h))


def _run_pair(kind, n, nrays, axis, ib, project, n_saves, jitter, precision):
    ne, rays, origin, spacing, omega = case(kind, n, nrays, axis=axis, jitter=jitter, seed=n + axis)
    sched = _sched(n, n_saves, n_saves == 1)
    Te, Z = (20.0, 1.0) if ib else (None, None)
    kw = dict(axis=axis, project=project, plane=L / 2, inv_brems=ib, Te=Te, Z=Z)
    k = run_kernel(ne, rays, origin, spacing, omega, sched, precision=precision, **kw)
    o = run_oracle(ne, rays, origin, spacing, omega, sched, **kw)
    return k, o


@pytest.mark.parametrize("kind,n,nrays,axis,ib,project,n_saves,jitter", CASES)
def test_trace_f64_matches_oracle(kind, n, nrays, axis, ib, project, n_saves, jitter):
    k, o = _run_pair(kind, n, nrays, axis, ib, project, n_saves, jitter, "f64")
    assert position_error(k["state"], o["state"], L) < 1e-10
    assert direction_error(k["state"], o["state"]) < 1e-10
    np.testing.assert_allclose(k["jones"][:, [0, 2]], o["jones"][:, [0, 2]], rtol=0, atol=1e-10 * L)
    np.testing.assert_allclose(k["jones"][:, [1, 3]], o["jones"][:, [1, 3]], rtol=0, atol=1e-10)
    ph = np.abs(o["phase"]).max()
    np.testing.assert_allclose(k["phase"], o["phase"], rtol=0, atol=1e-10 * max(ph, 1e-30))
    if ib:
        np.testing.assert_allclose(k["amp"], o["amp"], rtol=0, atol=1e-12)
    assert (k["steps"] != o["steps"]).mean() < 1e-3
    assert (k["status"] != o["status"]).mean() < 1e-3
    assert k["total_steps"] == int(k["steps"].astype(np.int64).sum())


def side_exit(state_last, axis):
    """Rays whose transverse position at the last save is outside the box."""
    t = [a for a in range(3) if a != axis]
    return (np.abs(state_last[t[0]]) > L / 2) | (np.abs(state_last[t[1]]) > L / 2)


@pytest.mark.parametrize("kind,n,nrays,axis,ib,project,n_saves,jitter", CASES)
def test_trace_f32_within_tolerance(kind, n, nrays, axis, ib, project, n_saves, jitter):
    k, o = _run_pair(kind, n, nrays, axis, ib, project, n_saves, jitter, "f32")
    pe = position_error(k["state"], o["state"], L)
    de = direction_error(k["state"], o["state"])
    assert pe < 1e-6, pe
    assert de < 1e-6, de
    side = side_exit(o["state"][-1], axis)
    ph = max(np.abs(o["phase"]).max(), 1e-30)
    dph = np.abs(k["phase"] - o["phase"])
    assert dph[:, ~side].max() <= 1e-6 * ph, dph[:, ~side].max() / ph
    assert dph.max() <= 1e-3 * ph
    if ib:
        damp = np.abs(k["amp"].astype(np.float64) - o["amp"])
        assert damp[:, ~side].max() < 1e-6, damp[:, ~side].max()
        assert damp.max() < 1e-4
    assert (k["steps"] != o["steps"]).mean() < 5e-3


def test_order_invariance_bitwise():
    """Each ray's result is independent of the order and company it is traced in."""
    ne, rays, origin, spacing, omega = case("kolmogorov", 40, 4000, seed=11)
    sched = _sched(40, 3, False)
    a = run_kernel(ne, rays, origin, spacing, omega, sched, precision="f32", inv_brems=True, Te=20.0, Z=1.0)
    perm = np.random.RandomState(0).permutation(rays.shape[1])
    sub = perm[:1234]
    b = run_kernel(ne, np.ascontiguousarray(rays[:, sub]), origin, spacing, omega, sched, precision="f32",
                   inv_brems=True, Te=20.0, Z=1.0)
    for key in ("jones", "state", "phase", "amp"):
        np.testing.assert_array_equal(b[key][..., :], a[key][..., sub])
    np.testing.assert_array_equal(b["steps"], a["steps"][sub])


def test_rays_starting_outside():
    """Rays outside the grid: receding ones leave at once, approaching ones drift in."""
    ne, rays, origin, spacing, omega = case("sinusoid", 32, 8)
    rays = rays.astype(np.float64)
    rays[0, 0] = 3e-3          # outside in x, moving along z only -> never enters
    rays[2, 1] = -4e-3         # 1.5 mm before the entry face -> drifts in
    rays[5, 2] = -C            # on the entry face moving backwards -> leaves at once
    rays[0, 3], rays[3, 3] = -2.6e-3, 0.01 * C   # outside in x, moving towards the grid
    rays[5, 3] = C * np.sqrt(1 - 0.01 ** 2)
    rays = rays.astype(np.float32)
    sched = _sched(32, 3, False)
    for precision in ("f64", "f32"):
        k = run_kernel(ne, rays, origin, spacing, omega, sched, precision=precision)
        o = run_oracle(ne, rays, origin, spacing, omega, sched)
        assert position_error(k["state"], o["state"], L) < (1e-10 if precision == "f64" else 1e-6)
        np.testing.assert_array_equal(k["steps"], o["steps"])
        assert k["steps"][0] == 0 and k["steps"][2] <= 1   # ray 2 leaves through a zero-length clipped step
        assert k["steps"][1] > 0


def test_empty_single_and_vacuum():
    ne, rays, origin, spacing, omega = case("vacuum", 16, 5)
    sched = _sched(16, 2, False)
    k = run_kernel(ne, rays, origin, spacing, omega, sched, precision="f32")
    np.testing.assert_allclose(k["state"][-1, :2], rays[:2], rtol=0, atol=1e-9)
    assert (k["phase"] == 0).all()
    one = run_kernel(ne, np.ascontiguousarray(rays[:, :1]), origin, spacing, omega, sched, precision="f64")
    assert one["jones"].shape == (2, 4, 1)
    g = runtime.pack_grid(torch.from_numpy(ne), origin, spacing, omega)
    out = runtime.trace(g, torch.zeros((6, 0), device="cuda"), sched)
    torch.cuda.synchronize()
    assert out["jones"].shape == (2, 4, 0) and int(out["total_steps"][0]) == 0


def test_error_codes_from_device_entry_points():
    ne, rays, origin, spacing, omega = case("sinusoid", 16, 64)
    g = runtime.pack_grid(torch.from_numpy(ne), origin, spacing, omega)
    r = torch.from_numpy(rays).cuda()
    sched = _sched(16, 1, True)
    small = torch.empty(1024, dtype=torch.uint8, device="cuda")
    with pytest.raises(_capi.SlothError) as e:
        runtime.trace(g, r, sched, workspace=small)
    assert e.value.code == _capi.SLOTH_ERR_WORKSPACE_TOO_SMALL
    bad = torch.empty(g.data.numel() + 4, dtype=torch.float32, device="cuda")[1:]
    with pytest.raises(_capi.SlothError) as e:
        runtime.pack_grid(torch.from_numpy(ne), origin, spacing, omega, out=bad)
    assert e.value.code == _capi.SLOTH_ERR_MISALIGNED


def _noncubic_case(axis, nrays=2000, seed=3):
    """A (72, 40, 56)-point grid over 6 x 4 x 5 mm (three spacings), a smooth
    density with structure on every axis, rays entering through the low face
    of `axis` with 1 mrad of jitter."""
    n = (72, 40, 56)
    ext = (6e-3, 4e-3, 5e-3)
    h = tuple(e / (k - 1) for e, k in zip(ext, n))
    origin = tuple(-e / 2 for e in ext)
    c = [origin[a] + h[a] * np.arange(n[a]) for a in range(3)]
    X, Y, Z = np.meshgrid(*c, indexing="ij")
    ne = (1e25 * (1 + 0.2 * np.sin(2 * np.pi * X / 1.3e-3) * np.cos(2 * np.pi * Y / 0.9e-3)
                  + 0.15 * np.sin(2 * np.pi * Z / 1.7e-3 + 0.4))).astype(np.float32)
    rng = np.random.RandomState(seed)
    rays = np.zeros((6, nrays), np.float32)
    for a in range(3):
        if a == axis:
            rays[a] = origin[a]
        else:
            rays[a] = rng.normal(0, ext[a] / 6, nrays)
    d = np.zeros((3, nrays))
    d[axis] = 1.0
    for a in range(3):
        if a != axis:
            d[a] = rng.normal(0, 1e-3, nrays)
    d /= np.linalg.norm(d, axis=0)
    rays[3:] = (d * C).astype(np.float32)
    sched = runtime.schedule_times(np.linspace(0.0, ext[axis], 3), h)
    return ne, rays, origin, h, 2 * np.pi * C / 532e-9, sched, ext


@pytest.mark.parametrize("axis", [0, 1])
@pytest.mark.parametrize("integ", ["rkn", "rk4"])
def test_noncubic_anisotropic_grid(axis, integ):
    ne, rays, origin, h, omega, sched, ext = _noncubic_case(axis)
    kw = dict(axis=axis, project=True, plane=ext[axis] / 2, inv_brems=True, Te=20.0, Z=1.0, integrator=integ)
    o = run_oracle(ne, rays, origin, h, omega, sched, **kw)
    k64 = run_kernel(ne, rays, origin, h, omega, sched, precision="f64", **kw)
    Lmax = max(ext)
    assert position_error(k64["state"], o["state"], Lmax) < 1e-10
    assert direction_error(k64["state"], o["state"]) < 1e-10
    np.testing.assert_allclose(k64["phase"], o["phase"], rtol=0, atol=1e-10 * np.abs(o["phase"]).max())
    np.testing.assert_allclose(k64["amp"], o["amp"], rtol=0, atol=1e-12)
    k32 = run_kernel(ne, rays, origin, h, omega, sched, precision="f32", **kw)
    assert position_error(k32["state"], o["state"], Lmax) < 1e-6
    assert direction_error(k32["state"], o["state"]) < 1e-6
    t = [a for a in range(3) if a != axis]
    far = (np.abs(o["state"][-1][t[0]]) <= ext[t[0]] / 2) & (np.abs(o["state"][-1][t[1]]) <= ext[t[1]] / 2)
    assert far.mean() > 0.9
    ph = np.abs(o["phase"]).max()
    assert np.abs(k32["phase"] - o["phase"])[:, far].max() <= 1e-6 * ph
    assert np.abs(k32["amp"].astype(np.float64) - o["amp"])[:, far].max() < 1e-6


@pytest.mark.parametrize("integ", ["rkn", "rk4"])
@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_interior_fast_path_is_bitwise_identical(precision, integ):
    """With a known density range the tracer skips the per-stage grid test on
    interior steps, the face test on runs of steps proven interior, and the
    warp's per-step bookkeeping while all its rays are on such a run. It takes
    the same kind of step in every case, so the FP32 results must not change
    at all. The FP64 kernels are compiled from the same source, but the
    compiler fuses multiplies and adds differently in the fast kernel's step
    loop, so FP64 is held to 1e-12 relative (measured 5e-13 on positions);
    each FP64 ray is still bitwise reproducible (order, chunking and serving
    tests)."""
    import dataclasses
    ne, rays, origin, spacing, omega = case("kolmogorov", 48, 3000, seed=21, jitter=2e-3)
    sched = _sched(48, 3, False)
    g = runtime.pack_grid(torch.from_numpy(ne), origin, spacing, omega, precision=precision)
    assert g.q_min <= 0.0 < g.q_max
    dt = torch.float32 if precision == "f32" else torch.float64
    r = torch.from_numpy(rays).to("cuda", dt)
    kw = dict(project=True, plane=L / 2, inv_brems=True, Te=20.0, Z=1.0, want_state=True, integrator=integ)
    fast = runtime.trace(g, r, sched, **kw)
    slow = runtime.trace(dataclasses.replace(g, q_min=float("inf")), r, sched, **kw)
    torch.cuda.synchronize()
    for key in ("jones", "state", "phase", "amp", "status", "steps", "total_steps"):
        if precision == "f32" or key in ("status", "steps", "total_steps"):
            assert torch.equal(fast[key], slow[key]), key
        else:
            f, s_ = fast[key].double(), slow[key].double()
            scale = s_.abs().amax(dim=-1, keepdim=True).clamp_min(1e-300)
            assert float(((f - s_).abs() / scale).max()) < 1e-12, key


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_dense_plasma_interior_runs(precision):
    """A density near 0.4 nc bounds the accelerations above the interior
    sampling limit (0.03 cells per step^2), so the tracer keeps the grid test
    on every stage but still skips the face test on runs of steps proven
    interior. The results must equal the kernel without any fast path (FP32
    bitwise, FP64 to rounding) and the oracle."""
    import dataclasses
    n = 48
    h = L / (n - 1)
    ne = workloads.kolmogorov_box(n, L=L, mean=1.5e27, rms=0.2, seed=51).numpy()
    rays = workloads.gaussian_beam(3000, waist=1.5e-3, L=L, seed=52, jitter=2e-3).numpy()
    omega = 2 * np.pi * C / 532e-9
    sched = _sched(n, 3, False)
    g = runtime.pack_grid(torch.from_numpy(ne), (-L / 2,) * 3, (h,) * 3, omega, precision=precision)
    bound = 0.5 * (sched.dtau / h) ** 2 * (g.q_max - min(g.q_min, 0.0))
    assert 0.03 < bound < 1.0
    dt = torch.float32 if precision == "f32" else torch.float64
    r = torch.from_numpy(rays).to("cuda", dt)
    kw = dict(project=True, plane=L / 2, inv_brems=True, Te=20.0, Z=1.0, want_state=True)
    runs = runtime.trace(g, r, sched, **kw)
    plain = runtime.trace(dataclasses.replace(g, q_min=float("inf")), r, sched, **kw)
    torch.cuda.synchronize()
    for key in ("jones", "state", "phase", "amp", "status", "steps", "total_steps"):
        if precision == "f32" or key in ("status", "steps", "total_steps"):
            assert torch.equal(runs[key], plain[key]), key
        else:
            f, s_ = runs[key].double(), plain[key].double()
            scale = s_.abs().amax(dim=-1, keepdim=True).clamp_min(1e-300)
            assert float(((f - s_).abs() / scale).max()) < 1e-12, key
    k = {kk: v.cpu().numpy() for kk, v in runs.items()}
    o = run_oracle(ne, rays, (-L / 2,) * 3, (h,) * 3, omega, sched, **{kk: kw[kk] for kk in ("project", "plane", "inv_brems", "Te", "Z")})
    tol = 1e-10 if precision == "f64" else 1e-6
    assert position_error(k["state"], o["state"], L) < tol
    assert direction_error(k["state"], o["state"]) < tol


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_nonfinite_rays_are_flagged_and_leave_the_others_unchanged(precision):
    """Rays whose position or direction holds NaN or Inf end with status
    SLOTH_RAY_NONFINITE and non-finite outputs. The finite rays traced in the
    same launch get bitwise the results they get without them. (The Morton
    keys clamp such coordinates into the grid, and the samplers' index clamps
    keep every grid access inside it, so these rays only waste their steps.)"""
    ne, rays, origin, spacing, omega = case("kolmogorov", 40, 512, seed=5)
    sched = _sched(40, 3, False)
    dt = torch.float32 if precision == "f32" else torch.float64
    bad = rays.astype(np.float64)
    picks = {3: (0, np.nan), 17: (4, np.nan), 64: (2, np.inf), 100: (1, -np.inf), 200: (5, np.inf),
             300: (3, -np.inf)}
    for ray, (row, value) in picks.items():
        bad[row, ray] = value
    idx = np.array(sorted(picks))
    good = np.setdiff1d(np.arange(rays.shape[1]), idx)
    g = runtime.pack_grid(torch.from_numpy(ne), origin, spacing, omega, precision=precision)
    kw = dict(inv_brems=True, Te=20.0, Z=1.0, want_state=True, want_status=True, want_steps=True)
    mixed = runtime.trace(g, torch.from_numpy(bad).to("cuda", dt), sched, **kw)
    alone = runtime.trace(g, torch.from_numpy(np.ascontiguousarray(bad[:, good])).to("cuda", dt), sched, **kw)
    torch.cuda.synchronize()
    m = {k: v.cpu().numpy() for k, v in mixed.items()}
    a = {k: v.cpu().numpy() for k, v in alone.items()}
    assert (m["status"][idx] == _capi.SLOTH_RAY_NONFINITE).all(), m["status"][idx]
    assert (m["status"][good] != _capi.SLOTH_RAY_NONFINITE).all()
    assert not np.isfinite(m["state"][-1][:, idx]).all(axis=0).any()
    for key in ("jones", "state", "phase", "amp"):
        if precision == "f32":
            np.testing.assert_array_equal(m[key][..., good], a[key])
        else:   # FP64 is held to 1e-12 of the output's scale, as in the fast-path test
            scale = np.abs(a[key]).max()
            assert np.abs(m[key][..., good] - a[key]).max() <= 1e-12 * scale, key
    np.testing.assert_array_equal(m["status"][good], a["status"])
    np.testing.assert_array_equal(m["steps"][good], a["steps"])
    # every ray, finite or not, stops at the last save
    assert m["steps"].max() <= sched.last_step


@pytest.mark.parametrize("shape", [(2, 2, 2), (2, 3, 5), (5, 2, 3)])
def test_smallest_grids(shape):
    """Grids of two points on some axes (one cell; the smallest the ABI
    takes): the cell index clamps to 0, the one-sided gradients of the pack
    are the only ones, and no interior run fits. FP64 and FP32 against the
    oracle with the module's tolerances."""
    rng = np.random.RandomState(sum(shape))
    ne = (1e25 * (1.0 + 0.3 * rng.rand(*shape))).astype(np.float32)
    h = tuple(L / (n - 1) for n in shape)
    origin = (-L / 2,) * 3
    omega = 2 * np.pi * C / 532e-9
    rays = workloads.gaussian_beam(500, waist=1.5e-3, L=L, seed=3).numpy()
    sched = runtime.schedule_times(np.linspace(0.0, L, 3), h)
    kw = dict(inv_brems=True, Te=20.0, Z=1.0)
    o = run_oracle(ne, rays, origin, h, omega, sched, **kw)
    k64 = run_kernel(ne, rays, origin, h, omega, sched, precision="f64", **kw)
    assert position_error(k64["state"], o["state"], L) < 1e-10
    assert direction_error(k64["state"], o["state"]) < 1e-10
    np.testing.assert_allclose(k64["phase"], o["phase"], rtol=0, atol=1e-10 * np.abs(o["phase"]).max())
    np.testing.assert_allclose(k64["amp"], o["amp"], rtol=0, atol=1e-12)
    np.testing.assert_array_equal(k64["steps"], o["steps"])
    k32 = run_kernel(ne, rays, origin, h, omega, sched, precision="f32", **kw)
    assert position_error(k32["state"], o["state"], L) < 1e-6
    assert direction_error(k32["state"], o["state"]) < 1e-6
    far = (np.abs(o["state"][-1][0]) <= L / 2) & (np.abs(o["state"][-1][1]) <= L / 2)
    assert far.mean() > 0.9
    assert np.abs(k32["phase"] - o["phase"])[:, far].max() <= 1e-6 * np.abs(o["phase"]).max()
    assert np.abs(k32["amp"].astype(np.float64) - o["amp"])[:, far].max() < 1e-6


@pytest.mark.parametrize("precision,rtol", [("f64", 1e-12), ("f32", 1e-6)])
@pytest.mark.parametrize("name", ["smooth_532", "dense_1064", "holes_532"])
def test_trace_layout_phase_channel_matches_reference_phase(name, precision, rtol):
    """K1's trace layout on the device, sampled by K0 at the golden points:
    omega times the interpolated n - 1 channel is the legacy solver's own
    ScalarDomain.phase (src/legacy/full_solver.py:342-345), 0 outside."""
    g = golden("phase")
    ne, pts, ref = g[f"{name}_ne"], g[f"{name}_points"], g[f"{name}_phase"]
    ax = [g[f"{name}_{a}"] for a in "xyz"]
    omega = float(g[f"{name}_omega"])
    grid = runtime.pack_grid(torch.from_numpy(ne), [a[0] for a in ax], [a[1] - a[0] for a in ax], omega,
                             precision=precision)
    got = omega * runtime.sample(grid, pts)[0].cpu().numpy().astype(np.float64)
    assert np.abs(got - ref).max() <= rtol * np.abs(ref).max()
