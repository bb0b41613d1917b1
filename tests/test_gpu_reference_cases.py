"""The reference's own test cases (tests/test_quadratic_trough.py of SLOTH),
run through this package's public API on the GPU, against the analytic
answers those tests use and against golden outputs of the reference's own
trace_and_save_depths / solve (tests/golden/make_golden.py)."""
import os
import pickle
import tempfile
import types
import warnings

import numpy as np
import pytest

from conftest import golden
from sloth_b200.core import physics
from sloth_b200.core.domain import ScalarDomain
from sloth_b200.core.propagator import (dsdt, kappa_inv_brems, precompute_gradients, solve,
                                        trace_and_save_depths)

pytestmark = pytest.mark.gpu

c = physics.C
_ALPHA = 3.14207787e-4
_LWL = 1064e-9
_OMEGA = 2 * np.pi * c / _LWL
_A, _HALF_Z, _DEPTH_MAX = 5e-3, 11e-3, 20e-3
_ANGLE = np.pi / 4.0
_OMEGA_OSC = _ANGLE / (_DEPTH_MAX / c)
_NE_0 = (_OMEGA_OSC * _A * np.sqrt(_ALPHA) * _OMEGA / c) ** 2
_X0 = np.array([0.5e-3, 1.0e-3, 1.5e-3, 2.0e-3])


def _trough(n_xy=24, n_z=24, inv_brems=False, Te=None, Z=None):
    x = np.linspace(-_A, _A, n_xy)
    z = np.linspace(-_HALF_Z, _HALF_Z, n_z)
    XX, _, _ = np.meshgrid(x, x, z, indexing='ij')
    d = types.SimpleNamespace()
    d.ne = (_NE_0 * (XX / _A) ** 2).astype(np.float32)
    d.x = x.astype(np.float32)
    d.y = x.astype(np.float32)
    d.z = z.astype(np.float32)
    d.probing_direction = 'z'
    d.lengths = np.array([x[-1] - x[0], x[-1] - x[0], z[-1] - z[0]], dtype=np.float32)
    d.dims = np.array([n_xy, n_xy, n_z], dtype=np.int32)
    d.Np_total = None
    d.inv_brems = inv_brems
    d.Te = None if Te is None else np.float32(Te)
    d.Z = None if Z is None else np.float32(Z)
    return d


def _rays(x0, z_start):
    s0 = np.zeros((6, len(x0)))
    s0[0] = x0
    s0[2] = z_start
    s0[5] = c
    return s0.astype(np.float32)


@pytest.mark.parametrize("precision,pos_tol", [("f64", 3e-9), ("f32", 1e-8)])
def test_trough_matches_analytic_and_reference(precision, pos_tol):
    t = golden("trace_cases")
    r = trace_and_save_depths(_rays(_X0, -_HALF_Z), _trough(), step=_DEPTH_MAX, depth_max=_DEPTH_MAX,
                              output_path=None, lwl=_LWL, jones_components=None, verbose=False, precision=precision)
    jv = np.asarray(r['jvec'][-1], dtype=np.float64)
    np.testing.assert_allclose(jv[0], _X0 * np.cos(_ANGLE), atol=0.2e-3)           # reference test tolerance
    np.testing.assert_allclose(jv[0], _X0 * np.cos(_ANGLE), atol=pos_tol)           # this build
    np.testing.assert_allclose(jv[[0, 2]], t["trough_jvec"][-1][[0, 2]], atol=pos_tol)
    np.testing.assert_allclose(jv[1] * c, -_X0 * _OMEGA_OSC * np.sin(_ANGLE), rtol=0.10)
    np.testing.assert_allclose(jv[2], 0.0, atol=0.1e-3)


def test_vacuum_straight_rays():
    n, half = 16, 2e-3
    coords = np.linspace(-half, half, n)
    d = types.SimpleNamespace(ne=np.zeros((n, n, n), np.float32), x=coords.astype(np.float32),
                              y=coords.astype(np.float32), z=coords.astype(np.float32), probing_direction='z',
                              lengths=np.array([2 * half] * 3, np.float32), dims=np.array([n] * 3, np.int32),
                              Np_total=None, inv_brems=False)
    x0 = np.array([0.5e-3, 1.0e-3])
    r = trace_and_save_depths(_rays(x0, -half), d, step=2 * half, depth_max=2 * half, output_path=None,
                              lwl=_LWL, jones_components=[0], verbose=False)
    np.testing.assert_allclose(np.asarray(r['jvec'][-1][0], np.float64), x0, atol=1e-6)


def _brems_run(precision="f32"):
    return trace_and_save_depths(_rays(_X0, -_HALF_Z), _trough(20, 20, True, 100.0, 1.0), step=_DEPTH_MAX / 4,
                                 depth_max=_DEPTH_MAX, output_path=None, lwl=_LWL, jones_components=[0, 1],
                                 verbose=False, precision=precision)


def test_brems_geometry_amplitude_and_reference():
    t = golden("trace_cases")
    r = _brems_run()
    np.testing.assert_allclose(r['jvec'][-1][0], _X0 * np.cos(_ANGLE), atol=0.2e-3)
    amps = [float(np.asarray(a).mean()) for a in r['amplitude']]
    assert amps[-1] < 1.0
    assert all(amps[i] <= amps[i - 1] + 1e-6 for i in range(1, len(amps)))
    # against the reference run (DOP853): the fixed-step quadrature of the piecewise
    # smooth kappa differs by ~1e-5 (see the oracle tests)
    np.testing.assert_allclose(np.stack(r['amplitude']), t["trough_ib_amp"], atol=2e-5)
    jv = np.asarray(r['jvec'][-1])
    amp = np.asarray(r['amplitude'][-1])
    assert np.sqrt(np.nanmean((jv * amp) ** 2)) <= np.sqrt(np.nanmean(jv ** 2)) + 1e-10


def test_geometry_identical_with_and_without_brems():
    rng = np.random.RandomState(0)
    x0 = _A * 0.3 * (rng.rand(30) - 0.5)
    kw = dict(step=_DEPTH_MAX, depth_max=_DEPTH_MAX, output_path=None, lwl=_LWL, jones_components=[0, 1],
              verbose=False)
    a = trace_and_save_depths(_rays(x0, -_HALF_Z), _trough(16, 16), **kw)
    b = trace_and_save_depths(_rays(x0, -_HALF_Z), _trough(16, 16, True, 100.0, 1.0), **kw)
    # the optical depth does not feed back into the trajectory: identical bits
    np.testing.assert_array_equal(a['jvec'][-1][0], b['jvec'][-1][0])


def _vacuum(half=2e-3, n=12):
    coords = np.linspace(-half, half, n)
    return types.SimpleNamespace(ne=np.zeros((n, n, n), np.float32), x=coords.astype(np.float32),
                                 y=coords.astype(np.float32), z=coords.astype(np.float32), probing_direction='z',
                                 lengths=np.array([2 * half] * 3, np.float32), dims=np.array([n] * 3, np.int32),
                                 Np_total=None, inv_brems=False)


def _small_rays(Np=8, z_start=-2e-3):
    s0 = np.zeros((6, Np))
    s0[0] = np.linspace(-5e-4, 5e-4, Np)
    s0[2] = z_start
    s0[5] = c
    return s0.astype(np.float32)


def _api(domain, **kw):
    d = dict(step=500e-6, depth_max=1e-3, output_path=None, lwl=1064e-9, verbose=False)
    d.update(kw)
    return trace_and_save_depths(_small_rays(), domain, **d)


def test_api_contracts():
    r = _api(_vacuum())
    assert set(r) == {'depth_saves', 'jvec', 'jones_components'}
    np.testing.assert_allclose(np.diff(_api(_vacuum(), step=200e-6)['depth_saves']), 200e-6, rtol=1e-6)
    with pytest.raises(ValueError, match="smaller than the requested depth_max"):
        _api(_vacuum(half=2e-3), depth_max=10e-3)
    full = _api(_vacuum())
    pos = _api(_vacuum(), jones_components='position')
    for j in range(len(full['jvec'])):
        np.testing.assert_array_equal(pos['jvec'][j], full['jvec'][j][[0, 2], :])
    with tempfile.NamedTemporaryFile(suffix='.pkl', delete=False) as f:
        path = f.name
    try:
        res = _api(_vacuum(), output_path=path)
        with open(path, 'rb') as fh:
            loaded = pickle.load(fh)
        np.testing.assert_array_equal(loaded['depth_saves'], res['depth_saves'])
        np.testing.assert_array_equal(loaded['jvec'][0], res['jvec'][0])
    finally:
        os.remove(path)
    assert 'amplitude' not in r and 'jvec_unweighted' not in r


def test_analytic_amplitude_and_reference():
    t = golden("trace_cases")
    ne_val, Te, Z, half, depth = 1e25, 100.0, 1.0, 3e-3, 2e-3
    coords = np.linspace(-half, half, 16)
    d = types.SimpleNamespace(ne=np.full((16, 16, 16), ne_val, np.float32), x=coords.astype(np.float32),
                              y=coords.astype(np.float32), z=coords.astype(np.float32), probing_direction='z',
                              lengths=np.array([2 * half] * 3, np.float32), dims=np.array([16] * 3, np.int32),
                              Np_total=None, inv_brems=True, Te=np.float32(Te), Z=np.float32(Z))
    kappa = float(kappa_inv_brems(np.float32(ne_val), np.float32(Te), Z, _OMEGA))
    r = trace_and_save_depths(t["uniform_s0"], d, step=500e-6, depth_max=depth, output_path=None, lwl=_LWL,
                              verbose=False)
    amp = np.stack(r['amplitude']).astype(np.float64)
    np.testing.assert_allclose(amp[-1].mean(), np.exp(-kappa * depth / c), rtol=0.05)
    np.testing.assert_allclose(amp, t["uniform_amp"], atol=1e-6)


@pytest.mark.parametrize("precision,tol", [("f64", 5e-9), ("f32", 2e-8)])
def test_solve_matches_reference(precision, tol):
    t = golden("trace_cases")
    d = _trough()
    d.region_count = 1
    d.ray_batch_count = 1
    rf, amp, duration = solve(t["trough_s0"], d, float(t["solve_depth"]), lwl=_LWL, verbose=False,
                              precision=precision)
    assert amp is None and duration >= 0
    np.testing.assert_allclose(np.asarray(rf, np.float64)[[0, 2]], t["solve_rf"][[0, 2]], atol=tol)
    np.testing.assert_allclose(np.asarray(rf, np.float64)[[1, 3]], t["solve_rf"][[1, 3]], atol=5e-8)


def test_solve_with_beam_tuple_and_extras():
    dom = ScalarDomain(5e-3, 32, ne_type="test_exponential_cos", Np=500)
    rf, amp, dur, ex = solve((1e-3, 1e-4, 2.5e-3, 'z', 'circular', True), dom, 5e-3, lwl=532e-9, verbose=False,
                             return_extras=True, detector_plane=2.5e-3)
    assert rf.shape == (4, 500) and amp is None
    assert ex["phase"].shape == (2, 500) and (ex["phase"][-1] <= 0).all()
    assert ex["total_steps"] == int(ex["steps"].sum())
    raw, _, _ = solve((1e-3, 1e-4, 2.5e-3, 'z', 'circular', True), dom, 5e-3, lwl=532e-9, verbose=False,
                      return_raw_results=True)
    assert raw[0].ys.shape == (500, 2, 6)


def test_precompute_gradients_and_dsdt_match_reference():
    g = golden("precompute_gradients")
    got = precompute_gradients(g["ne"], g["x"], g["y"], g["z"], float(g["omega"]))
    for k, name in enumerate(("dndx", "dndy", "dndz")):
        np.testing.assert_allclose(got[k], g[name], rtol=1e-11, atol=0)
    s = golden("dsdt")
    for k in range(0, s["states"].shape[1], 7):
        sp = dsdt(0.0, s["states"][:, k], True, *got, g["x"], g["y"], g["z"], None, None, s["kappa"])
        np.testing.assert_allclose(sp, s["sprime"][:, k], rtol=1e-11, atol=1e-300)


def test_overcritical_warning():
    coords = np.linspace(-3e-3, 3e-3, 8)
    ncr = _ALPHA * _OMEGA ** 2
    with warnings.catch_warnings(record=True) as caught:
        warnings.simplefilter("always")
        precompute_gradients(np.full((8, 8, 8), 1.5 * ncr, np.float32), coords, coords, coords, _OMEGA)
    assert len(caught) == 1 and issubclass(caught[0].category, UserWarning)
