"""Generate golden vectors by running the SLOTH reference's own code.

JAX, diffrax and equinox are not installable here, so the reference modules
are imported with small stand-ins:

* ``jax.numpy``  -> numpy (arrays gain the ``.at[idx].set(v)`` functional update);
* ``jax.jit``, ``equinox.filter_jit`` -> identity; ``jax.vmap`` -> a loop over axis 0;
* ``diffrax.diffeqsolve(Tsit5, PIDController, SaveAt(ts))`` -> scipy
  ``solve_ivp(method="DOP853")`` at tight tolerances evaluated at the save times.

Everything else -- precompute_gradients, kappa_inv_brems, the trilinear
interpolator, dsdt, ray_to_Jonesvector, Beam, trace_and_save_depths, solve --
is the reference's own code, unmodified, read from its source tree.

The diagnostics module also imports matplotlib and sympy, which are not
installed either; only their names are needed (`Matrix` is used by the
reference's unused `ray` helper), so they are empty stand-ins.

Usage (in a container that has the reference at /root/reference):
    python tests/golden/make_golden.py [/path/to/reference] [--only=diagnostics|--only=phase]
Writes tests/golden/*.npz. The fixtures are committed; nothing on a GPU box
or in the tests reads the reference tree.
"""
from __future__ import annotations

import os
import sys
import types

import numpy as np

_POS = [a for a in sys.argv[1:] if not a.startswith("--")]
REF = _POS[0] if _POS else "/root/reference"
ONLY = next((a.split("=", 1)[1] for a in sys.argv[1:] if a.startswith("--only=")), None)
OUT = os.path.dirname(os.path.abspath(__file__))


# ---------------------------------------------------------------------------
# numpy stand-in for jax.numpy with functional .at[] updates
# ---------------------------------------------------------------------------
class AtArray(np.ndarray):
    """ndarray with JAX's value semantics: .at[idx].set(v) and augmented
    assignments return new arrays instead of writing in place."""

    @property
    def at(self):
        return _AtIndexer(self)

    def __iadd__(self, o):
        return np.add(self, o)

    def __isub__(self, o):
        return np.subtract(self, o)

    def __imul__(self, o):
        return np.multiply(self, o)

    def __itruediv__(self, o):
        return np.true_divide(self, o)


class _AtIndexer:
    def __init__(self, arr):
        self.arr = arr

    def __getitem__(self, idx):
        return _AtSetter(self.arr, idx)


class _AtSetter:
    def __init__(self, arr, idx):
        self.arr, self.idx = arr, idx

    def set(self, v):
        out = np.array(self.arr, copy=True)
        out[self.idx] = v
        return out.view(AtArray)


def _wrap(obj):
    if callable(obj) and not isinstance(obj, type):
        def f(*a, **k):
            r = obj(*a, **k)
            return r.view(AtArray) if isinstance(r, np.ndarray) and not isinstance(r, AtArray) else r
        return f
    return obj


class FakeJnp(types.ModuleType):
    def __getattr__(self, name):
        return _wrap(getattr(np, name))


def _install_stubs():
    jnp = FakeJnp("jax.numpy")
    jax = types.ModuleType("jax")
    jax.numpy = jnp
    jax.Array = np.ndarray
    jax.jit = lambda f=None, **k: (f if f is not None else (lambda g: g))

    def vmap(f, in_axes=(0, None)):
        def g(xs, *rest):
            outs = [f(xs[i], *rest) for i in range(xs.shape[0])]
            sol = outs[0]
            return types.SimpleNamespace(ys=np.stack([o.ys for o in outs]),
                                         ts=np.stack([o.ts for o in outs]), t0=sol.t0, t1=sol.t1,
                                         stats={}, result=None)
        return g

    jax.vmap = vmap
    jax.block_until_ready = lambda x: x
    jax.devices = lambda *a: ["cpu"]
    jax.default_backend = lambda: "cpu"
    jax.device_put = lambda x, *a: x
    jax.config = types.SimpleNamespace(update=lambda *a, **k: None)
    jax.checkpoint = lambda f: f
    src = types.ModuleType("jax._src")
    dtypes = types.ModuleType("jax._src.dtypes")
    dtypes.can_cast = np.can_cast
    tree = types.ModuleType("jax._src.tree_util")
    tree.register_pytree_node = lambda *a, **k: None
    nputil = types.ModuleType("jax._src.numpy.util")
    nputil.check_arraylike = lambda *a, **k: None

    def promote_dtypes_inexact(*args):
        out = []
        for a in args:
            a = np.asarray(a)
            out.append(a if np.issubdtype(a.dtype, np.inexact) else a.astype(np.float64))
        return out
    nputil.promote_dtypes_inexact = promote_dtypes_inexact
    srcnp = types.ModuleType("jax._src.numpy")
    scipy_ = types.ModuleType("jax.scipy")
    interp = types.ModuleType("jax.scipy.interpolate")
    interp.RegularGridInterpolator = None
    for name, mod in {"jax": jax, "jax.numpy": jnp, "jax._src": src, "jax._src.dtypes": dtypes,
                      "jax._src.tree_util": tree, "jax._src.numpy": srcnp, "jax._src.numpy.util": nputil,
                      "jax.scipy": scipy_, "jax.scipy.interpolate": interp}.items():
        sys.modules[name] = mod

    eqx = types.ModuleType("equinox")
    eqx.Module = object
    eqx.filter_jit = lambda f: f
    sys.modules["equinox"] = eqx

    mpl = types.ModuleType("matplotlib")
    mpl.use = lambda *a, **k: None
    plt = types.ModuleType("matplotlib.pyplot")
    mpl.pyplot = plt
    sys.modules["matplotlib"] = mpl
    sys.modules["matplotlib.pyplot"] = plt

    # diffrax: scipy DOP853 at tight tolerance in place of Tsit5 + PIDController
    from scipy.integrate import solve_ivp
    dfx = types.ModuleType("diffrax")

    class Solution(types.SimpleNamespace):
        pass

    class ODETerm:
        def __init__(self, fn):
            self.fn = fn

    class SaveAt:
        def __init__(self, ts):
            self.ts = np.asarray(ts, dtype=np.float64)

    def diffeqsolve(term, solver, t0, t1, dt0, y0, args=None, saveat=None, stepsize_controller=None,
                    max_steps=None):
        y0 = np.asarray(y0, dtype=np.float64)
        ts = saveat.ts
        sol = solve_ivp(lambda t, y: np.asarray(term.fn(t, y, args), dtype=np.float64),
                        (float(t0), float(t1)), y0, method="DOP853", t_eval=ts, rtol=1e-12,
                        atol=np.where(np.arange(y0.size) < 3, 1e-15, 1e-6))
        if not sol.success:
            raise RuntimeError(sol.message)
        return Solution(ys=sol.y.T, ts=ts, t0=t0, t1=t1, stats={}, result=None)

    dfx.Solution = Solution
    dfx.ODETerm = ODETerm
    dfx.Tsit5 = lambda: None
    dfx.SaveAt = SaveAt
    dfx.PIDController = lambda **k: None
    dfx.diffeqsolve = diffeqsolve
    sys.modules["diffrax"] = dfx


def main():
    _install_stubs()
    sys.path.insert(0, os.path.join(REF, "src"))
    if ONLY == "diagnostics":
        diagnostics_golden()
        return
    if ONLY == "phase":
        phase_golden()
        return
    import core.interpolator as ci           # noqa: E402
    import core.propagator as cp             # noqa: E402
    import shared.propagation as sp          # noqa: E402
    from core.beam import Beam               # noqa: E402
    from scipy.constants import c            # noqa: E402

    rng = np.random.RandomState(1234)

    # 1. precompute_gradients on float64 and float32 inputs, non-cubic grid
    shape = (6, 7, 8)
    ne64 = rng.uniform(1e24, 5e25, size=shape)
    x = np.linspace(-1e-3, 1e-3, shape[0])
    y = np.linspace(-2e-3, 1.5e-3, shape[1])
    z = np.linspace(-0.5e-3, 2.5e-3, shape[2])
    omega = 2 * np.pi * c / 532e-9
    g64 = cp.precompute_gradients(ne64, x, y, z, omega)
    ne32 = ne64.astype(np.float32)
    g32 = cp.precompute_gradients(ne32, x.astype(np.float32), y.astype(np.float32), z.astype(np.float32), omega)
    np.savez(os.path.join(OUT, "precompute_gradients.npz"), ne=ne64, x=x, y=y, z=z, omega=omega,
             dndx=np.asarray(g64[0]), dndy=np.asarray(g64[1]), dndz=np.asarray(g64[2]),
             dndx32=np.asarray(g32[0]), dndy32=np.asarray(g32[1]), dndz32=np.asarray(g32[2]))

    # 2. kappa_inv_brems incl. an over-critical density
    omegas = np.array([2 * np.pi * c / 1064e-9, 2 * np.pi * c / 532e-9])
    cases = []
    for om in omegas:
        nc = 3.14207787e-4 * om ** 2
        for ne in (1e23, 1e25, 3e26, 0.5 * nc, 1.5 * nc, 4.0 * nc):
            for Te, Z in ((100.0, 1.0), (10.0, 4.0), (20.0, 1.0), (1000.0, 2.0)):
                cases.append((ne, Te, Z, om, float(cp.kappa_inv_brems(np.float64(ne), np.float64(Te), Z, om))))
    np.savez(os.path.join(OUT, "kappa.npz"), cases=np.array(cases))

    # 3. interpolator, incl. out-of-bounds, on-node and face points
    vals = rng.normal(size=shape)
    pts = np.stack([rng.uniform(-1.2e-3, 1.2e-3, 400), rng.uniform(-2.2e-3, 1.7e-3, 400),
                    rng.uniform(-0.7e-3, 2.7e-3, 400)], axis=1)
    nodes = np.stack([x[[0, 2, 5, 5, 3]], y[[0, 6, 3, 1, 6]], z[[7, 0, 4, 7, 2]]], axis=1)
    pts = np.concatenate([pts, nodes])
    res = ci.RegularGridInterpolator((x, y, z), vals, pts, fill_value=0.0)
    np.savez(os.path.join(OUT, "interpolator.npz"), x=x, y=y, z=z, values=vals, points=pts,
             result=np.asarray(res))

    # 4. dsdt at random 7-states
    kap = cp.kappa_inv_brems(ne64, 50.0, 1.0, omega)
    states = np.stack([pts[:50, 0], pts[:50, 1], pts[:50, 2], rng.normal(0, 1e6, 50),
                       rng.normal(0, 1e6, 50), np.full(50, c), np.zeros(50)], axis=0)
    sp_out = []
    for k in range(states.shape[1]):
        sp_out.append(np.asarray(cp.dsdt(0.0, states[:, k], True, *g64, x, y, z, None, None, kap)))
    np.savez(os.path.join(OUT, "dsdt.npz"), states=states, kappa=np.asarray(kap), sprime=np.stack(sp_out, 1))

    # 5. ray_to_Jonesvector / back_propogate
    rays = np.stack([rng.normal(0, 1e-3, 20), rng.normal(0, 1e-3, 20), rng.normal(0, 1e-3, 20),
                     rng.normal(0, 3e5, 20), rng.normal(0, 3e5, 20), np.full(20, c * 0.999)])
    rays[3:, :5] = rays[[4, 5, 3], :5]  # a few rays with a large component on other axes
    jv = {}
    for d in "xyz":
        for keep in (True, False):
            jv[f"{d}_{int(keep)}"] = np.asarray(sp.ray_to_Jonesvector(rays, ne_extent=1.5e-3, probing_direction=d,
                                                                      keep_current_plane=keep)[0])
        jv[f"bp_{d}"] = np.asarray(sp.back_propogate(rays.view(AtArray), 1.5e-3, d))
    np.savez(os.path.join(OUT, "jones.npz"), rays=rays, **jv)

    # 6. Beam (seeded) for every implemented beam type and direction
    beams = {}
    # ('linear' is not included: the reference raises UnboundLocalError for it,
    # src/core/beam.py:238-254 never binds u or phi before the `del` at :338-341.)
    for bt, size in (("circular", 1e-3), ("square", 1e-3), ("rectangular", [1e-3, 2e-3]),
                     ("rect_trackers", [1e-3, 2e-3])):
        for d in "xyz":
            b = Beam(37, size, 2e-4, 2.5e-3, probing_direction=d, beam_type=bt, seeded=True)
            beams[f"{bt}_{d}"] = np.asarray(b.s0, dtype=np.float64)
    np.savez(os.path.join(OUT, "beam.npz"), **beams)

    # 7. trace_and_save_depths end to end (reference test cases) and solve()
    tr = _trace_cases(cp, c)
    np.savez(os.path.join(OUT, "trace_cases.npz"), **tr)
    diagnostics_golden()
    phase_golden()
    print("golden vectors written to", OUT)


def phase_golden():
    """The phase integrand of the legacy full solver, ScalarDomain.phase
    (src/legacy/full_solver.py:342-345): omega * (interp(n)(x) - 1), with n
    the refractive index on the grid points (:292-296, NRL omega_pe :236-239)
    and the interpolator's fill value 1.0 outside the grid (:289).

    The module imports only numpy and scipy, so it runs as shipped except for
    one defect: omega_pe is declared without `self` (:236) while n_refrac and
    kappa call it as a method, which raises TypeError. Binding it as a
    staticmethod fixes that call and changes nothing else.

    The grids have a power-of-two spacing with half-integer or integer
    offsets, so the float32 coordinates the legacy domain keeps (:118) are
    exactly the uniform float64 ones."""
    sys.path.insert(0, os.path.join(REF, "src", "legacy"))
    import full_solver as fs                 # noqa: E402
    from scipy.constants import c            # noqa: E402
    fs.ScalarDomain.omega_pe = staticmethod(fs.ScalarDomain.omega_pe)
    rng = np.random.RandomState(2718)
    h = 2.0 ** -13                           # 122 um
    out = {}
    for name, shape, lwl, dens in (("smooth_532", (9, 10, 11), 532e-9, "smooth"),
                                   ("dense_1064", (8, 7, 9), 1064e-9, "dense"),
                                   ("holes_532", (10, 8, 8), 532e-9, "holes")):
        coords = [(np.arange(m) - (m - 1) / 2.0) * h for m in shape]
        omega = 2 * np.pi * c / lwl
        nc = 3.14207787e-4 * omega ** 2
        if dens == "smooth":
            ne = rng.uniform(1e24, 5e25, size=shape)
        elif dens == "dense":
            ne = rng.uniform(0.1, 0.9, size=shape) * nc
        else:
            ne = rng.uniform(1e24, 5e25, size=shape) * (rng.uniform(size=shape) > 0.3)
        dom = fs.ScalarDomain(*coords, float(coords[0][-1]), phaseshift=True)
        dom.external_ne(ne)
        dom.calc_dndr(lwl)
        lo = np.array([a[0] for a in coords])
        hi = np.array([a[-1] for a in coords])
        inside = lo[:, None] + (hi - lo)[:, None] * rng.uniform(size=(3, 300))
        around = lo[:, None] - 0.1 * (hi - lo)[:, None] + 1.2 * (hi - lo)[:, None] * rng.uniform(size=(3, 100))
        idx = [rng.randint(0, m, 12) for m in shape]
        nodes = np.stack([coords[a][idx[a]] for a in range(3)])
        faces = inside[:, :12].copy()
        for k in range(12):
            faces[k % 3, k] = (lo if k % 2 else hi)[k % 3]
        pts = np.concatenate([inside, around, nodes, faces], axis=1)
        out[f"{name}_ne"] = ne
        out[f"{name}_x"], out[f"{name}_y"], out[f"{name}_z"] = coords
        out[f"{name}_omega"] = np.float64(dom.omega)
        out[f"{name}_points"] = pts
        out[f"{name}_phase"] = np.asarray(dom.phase(pts), dtype=np.float64)
    np.savez(os.path.join(OUT, "phase.npz"), **out)
    print("phase golden vectors written to", OUT)


def _trough_domain(c, ne_0, a, half_z, n_xy, n_z, inv_brems=False, Te=None, Z=None):
    xs = np.linspace(-a, a, n_xy)
    zs = np.linspace(-half_z, half_z, n_z)
    XX, _, _ = np.meshgrid(xs, xs, zs, indexing="ij")
    d = types.SimpleNamespace()
    d.ne = (ne_0 * (XX / a) ** 2).astype(np.float32)
    d.x = xs.astype(np.float32)
    d.y = xs.astype(np.float32)
    d.z = zs.astype(np.float32)
    d.probing_direction = "z"
    d.lengths = np.array([xs[-1] - xs[0], xs[-1] - xs[0], zs[-1] - zs[0]], dtype=np.float32)
    d.dims = np.array([n_xy, n_xy, n_z], dtype=np.int32)
    d.Np_total = None
    d.inv_brems = inv_brems
    d.Te = None if Te is None else np.float32(Te)
    d.Z = None if Z is None else np.float32(Z)
    d.region_count = 1
    d.ray_batch_count = 1
    return d


def _trace_cases(cp, c):
    """The reference test module's physics cases, run through the reference's
    own trace_and_save_depths / solve (DOP853 in place of Tsit5)."""
    lwl = 1064e-9
    omega = 2 * np.pi * c / lwl
    A, HALF_Z, DEPTH = 5e-3, 11e-3, 20e-3
    omega_osc = (np.pi / 4) / (DEPTH / c)
    ne_0 = (omega_osc * A * np.sqrt(3.14207787e-4) * omega / c) ** 2
    x0 = np.array([0.5e-3, 1.0e-3, 1.5e-3, 2.0e-3])
    s0 = np.zeros((6, 4))
    s0[0] = x0
    s0[2] = -HALF_Z
    s0[5] = c
    s0 = s0.astype(np.float32).view(AtArray)
    out = {"trough_s0": np.asarray(s0), "trough_ne0": ne_0}
    d = _trough_domain(c, ne_0, A, HALF_Z, 24, 24)
    r = cp.trace_and_save_depths(s0, d, step=DEPTH, depth_max=DEPTH, output_path=None, lwl=lwl,
                                 jones_components=None, verbose=False)
    out["trough_depths"] = r["depth_saves"]
    out["trough_jvec"] = np.stack(r["jvec"])
    d = _trough_domain(c, ne_0, A, HALF_Z, 20, 20, inv_brems=True, Te=100.0, Z=1.0)
    r = cp.trace_and_save_depths(s0, d, step=DEPTH / 4, depth_max=DEPTH, output_path=None, lwl=lwl,
                                 jones_components=None, verbose=False)
    out["trough_ib_depths"] = r["depth_saves"]
    out["trough_ib_jvec"] = np.stack(r["jvec"])
    out["trough_ib_amp"] = np.stack(r["amplitude"])
    # uniform absorbing plasma (TestAbsorptionFormula.test_analytic_amplitude_match)
    n, half = 16, 3e-3
    coords = np.linspace(-half, half, n)
    u = types.SimpleNamespace(ne=np.full((n, n, n), 1e25, dtype=np.float32), x=coords.astype(np.float32),
                              y=coords.astype(np.float32), z=coords.astype(np.float32), probing_direction="z",
                              lengths=np.array([2 * half] * 3, dtype=np.float32),
                              dims=np.array([n] * 3, dtype=np.int32), Np_total=None, inv_brems=True,
                              Te=np.float32(100.0), Z=np.float32(1.0), region_count=1, ray_batch_count=1)
    s1 = np.zeros((6, 10))
    s1[0] = np.linspace(-5e-4, 5e-4, 10)
    s1[2] = -half
    s1[5] = c
    s1 = s1.astype(np.float32).view(AtArray)
    r = cp.trace_and_save_depths(s1, u, step=500e-6, depth_max=2e-3, output_path=None, lwl=lwl, verbose=False)
    out["uniform_s0"] = np.asarray(s1)
    out["uniform_depths"] = r["depth_saves"]
    out["uniform_jvec"] = np.stack(r["jvec"])
    out["uniform_amp"] = np.stack(r["amplitude"])
    # solve(): final state at t = sqrt(8)*depth/c, keep_current_plane=True
    d = _trough_domain(c, ne_0, A, HALF_Z, 24, 24)
    rf, amp, _ = cp.solve(s0, d, 2 * HALF_Z, lwl=lwl, verbose=False)
    out["solve_rf"] = np.asarray(rf)
    out["solve_depth"] = 2 * HALF_Z
    return out


def diagnostics_golden():
    """Ray-transfer-matrix diagnostics (src/processing/diagnostics.py): the
    reference's own solve methods, histograms and module-level optics on
    seeded Jones vectors (x, theta, y, phi), metres and radians."""
    sym = types.ModuleType("sympy")
    sym.Matrix = lambda *a, **k: np.asarray(*a)
    sys.modules.setdefault("sympy", sym)
    import processing.diagnostics as dg      # noqa: E402

    rng = np.random.RandomState(4321)
    N = 1500
    rf = np.stack([rng.normal(0, 2e-3, N), rng.normal(0, 5e-3, N), rng.normal(0, 1.5e-3, N),
                   rng.normal(0, 4e-3, N)]).astype(np.float32)
    rf[:, 7] = np.nan
    rf[0, 11] = np.nan
    rf[3, 19] = np.nan
    weights = rng.uniform(0.5, 1.0, N).astype(np.float32)
    out = {"rf": rf, "weights": weights}

    def run(name, cls, solve, init_kw, hist_kw, solve_kw=None, use_weights=True):
        d = cls(rf.copy(), weights=weights.copy() if use_weights else None, **init_kw)
        if solve is not None:
            getattr(d, solve)(**(solve_kw or {}))
        d.histogram(**hist_kw)
        out[f"{name}_H"] = np.asarray(d.H, dtype=np.float64)
        out[f"{name}_xedges"] = np.asarray(d.xedges)
        out[f"{name}_yedges"] = np.asarray(d.yedges)
        out[f"{name}_rf"] = np.asarray(d.rf, dtype=np.float64)

    run("shadow_single", dg.Shadowgraphy, "single_lens_solve", dict(L=400, R=25, Lx=18, Ly=13.5),
        dict(bin_scale=16))
    run("shadow_two", dg.Shadowgraphy, "two_lens_solve", dict(focal_plane=1.0, L=400, R=25, Lx=18, Ly=13.5),
        dict(bin_scale=8), use_weights=False)
    run("shadow_custom", dg.Shadowgraphy, "single_lens_custom_solve",
        dict(L=400, R=25, Lx=18, Ly=13.5, prefilter_input=True, ccd_shape_m=(10e-3, 8e-3)),
        dict(bin_scale=12), solve_kw=dict(f=150, obj_dist=300, img_dist=600))
    run("schlieren_df", dg.Schlieren, "DF_solve", dict(L=400, R=25, Lx=18, Ly=13.5), dict(bin_scale=16),
        solve_kw=dict(R=1.0))
    run("schlieren_lf", dg.Schlieren, "LF_solve", dict(L=400, R=25, Lx=18, Ly=13.5), dict(bin_scale=16),
        solve_kw=dict(R=1.0))
    run("refract", dg.Refractometry, "incoherent_solve", dict(L=400, R=25, Lx=18, Ly=13.5), dict(bin_scale=16))
    run("refract_custom", dg.Refractometry, "incoherent_custom_solve", dict(L=400, R=25, Lx=18, Ly=13.5),
        dict(bin_scale=16), solve_kw=dict(f1=150, f3=250, img_f1_dist=500, img_dist=350))
    run("plain", dg.Shadowgraphy, None, dict(L=400, R=25, Lx=18, Ly=13.5), dict(bin_scale=16, plain_plot=True))
    # module-level optics on a mm copy of the first 400 rays
    r = dg.m_to_mm(rf[:, :400].astype(np.float64))
    out["op_in"] = r
    out["op_travel"] = dg.travel(r, 123.0)
    out["op_lens"] = dg.lens(r, 80.0, -120.0)
    out["op_circ_ap"] = dg.circular_aperture(r.copy(), 2.5)
    out["op_circ_stop"] = dg.circular_stop(r.copy(), 1.5)
    out["op_rect_ap"] = dg.rect_aperture(r.copy(), 2.0, 1.0)
    out["op_annular_mask"] = dg.annular_stop(r.copy(), 1.0, 2.5)
    out["op_knife_x_pos"] = dg.knife_edge(r.copy(), 0.5, "x", 1)
    out["op_knife_y_neg"] = dg.knife_edge(r.copy(), -0.25, "y", -1)
    out["op_lens_cutoff"] = dg.lens_cutoff(r.copy(), L=400, R=3)
    np.savez_compressed(os.path.join(OUT, "diagnostics.npz"), **out)
    print("diagnostics golden vectors written to", OUT)


if __name__ == "__main__":
    main()
