"""Host-side logic of the package, CPU only: Beam and ScalarDomain against the
reference, input validation that happens before any device call, the step
schedule, the host Jones projection and the synthetic workloads."""
import types

import numpy as np
import pytest
import torch

from conftest import golden
from sloth_b200 import runtime, workloads
from sloth_b200.core import physics
from sloth_b200.core.beam import Beam
from sloth_b200.core.domain import ScalarDomain
from sloth_b200.core.propagator import solve, trace_and_save_depths
from sloth_b200.shared import propagation as sp


def test_beam_matches_reference_golden():
    g = golden("beam")
    for key in g.files:
        bt, d = key.rsplit("_", 1)
        size = [1e-3, 2e-3] if bt in ("rectangular", "rect_trackers") else 1e-3
        s0 = Beam(37, size, 2e-4, 2.5e-3, probing_direction=d, beam_type=bt, seeded=True).s0
        assert s0.dtype == np.float32
        np.testing.assert_allclose(s0, g[key].astype(np.float32), rtol=2e-7, atol=1e-12 * 0 + 1e-30, err_msg=key)


def test_beam_errors_and_linear():
    with pytest.raises(AssertionError):
        Beam(4, [1e-3, 1e-3], 0.0, 1e-3, beam_type="circular")
    with pytest.raises(ValueError, match="unrecognised"):
        Beam(4, 1e-3, 0.0, 1e-3, beam_type="donut")
    with pytest.raises(NotImplementedError):
        Beam(4, 1e-3, 0.0, 1e-3, beam_type="even")
    lin = Beam(10, 1e-3, 1e-4, 1e-3, beam_type="linear", seeded=True).s0
    assert (lin[1] == 0).all() and (lin[4] == 0).all() and (np.abs(lin[0]) <= 1e-3).all()
    np.testing.assert_allclose(np.sqrt((lin[3:].astype(np.float64) ** 2).sum(0)), physics.C, rtol=1e-7)


def test_domain_validation_and_profiles():
    with pytest.raises(AssertionError, match="eV"):
        ScalarDomain([4e-3, 4e-3, 4e-3], [8, 8, 8], inv_brems=True, Te=-10.0, Z=1.0)
    with pytest.raises(AssertionError):
        ScalarDomain(4e-3, 8, inv_brems=True, Te=10.0)
    with pytest.raises(AssertionError):
        ScalarDomain(4e-3, 8, ne_type="nope")
    d = ScalarDomain(4e-3, [8, 9, 10], ne_type="test_slab")
    assert d.ne.shape == (8, 9, 10) and d.ne.dtype == np.float32
    assert d.x.dtype == np.float32 and d.x[0] == np.float32(-2e-3) and d.z.size == 10
    assert d.region_count == 1 and d.ray_batch_count == 1
    x = d.x.astype(np.float64)
    np.testing.assert_allclose(d.ne[:, 0, 0], 2e23 * (1 + x / 4e-3), rtol=1e-6)
    e = ScalarDomain(4e-3, 8, ne_type="test_exponential_cos")
    X, Y = np.meshgrid(e.x.astype(np.float64), e.y.astype(np.float64), indexing="ij")
    np.testing.assert_allclose(e.ne[:, :, 3], 1e24 * 10 ** (X / -2e-3) * (1 + np.cos(2 * np.pi * Y / 1e-3)),
                               rtol=1e-6, atol=1e18)
    assert ScalarDomain(4e-3, 8, ne_type="test_null").ne.max() == 0
    lc = ScalarDomain(4e-3, 8, ne_type="test_linear_cos")
    assert lc.ne.min() > 0


def _vacuum(half=2e-3, n=12):
    c1 = np.linspace(-half, half, n)
    return types.SimpleNamespace(ne=np.zeros((n, n, n), np.float32), x=c1.astype(np.float32),
                                 y=c1.astype(np.float32), z=c1.astype(np.float32), probing_direction='z',
                                 lengths=np.array([2 * half] * 3, np.float32), dims=np.array([n] * 3, np.int32),
                                 Np_total=None, inv_brems=False)


def test_trace_and_save_depths_validation_before_device():
    rays = np.zeros((6, 4), np.float32)
    kw = dict(output_path=None, verbose=False)
    with pytest.raises(ValueError, match="positive"):
        trace_and_save_depths(rays, _vacuum(), step=0.0, depth_max=1e-3, **kw)
    with pytest.raises(ValueError, match="smaller than the requested depth_max"):
        trace_and_save_depths(rays, _vacuum(), step=1e-4, depth_max=10e-3, **kw)
    with pytest.raises(ValueError, match="out of range"):
        trace_and_save_depths(rays, _vacuum(), step=1e-4, depth_max=1e-3, jones_components=[0, 5], **kw)
    with pytest.raises(AssertionError):
        trace_and_save_depths((1e-3, 0, 1e-3, 'z', 'circular', True), _vacuum(), step=1e-4, depth_max=1e-3, **kw)
    b = Beam(4, 1e-3, 0.0, 1e-3)
    with pytest.raises(AssertionError):
        solve(b, _vacuum(), 1e-3, verbose=False)


def test_schedule_lands_on_saves():
    h = (5e-3 / 511,) * 3
    s = runtime.schedule_times(np.linspace(0, 5e-3, 11), h)
    assert s.first_save == 0 and s.n_saves == 11
    assert s.dtau <= runtime.nominal_step(h) * (1 + 1e-12)
    np.testing.assert_allclose(s.dtau * s.save_every * np.arange(11), np.linspace(0, 5e-3, 11), rtol=1e-12)
    t = runtime.schedule_times([np.sqrt(8) * 5e-3], h)
    assert t.n_saves == 1 and t.first_save * t.dtau == pytest.approx(np.sqrt(8) * 5e-3, rel=1e-12)
    assert t.dtau <= runtime.nominal_step(h) * (1 + 1e-12)
    z = runtime.schedule_times([0.0], h)
    assert z.first_save == 0 and z.n_saves == 1
    with pytest.raises(NotImplementedError):
        runtime.uniform_axis([0.0, 1.0, 3.0])


def test_host_jones_matches_reference():
    g = golden("jones")
    for d in "xyz":
        for keep in (True, False):
            got, none = sp.ray_to_Jonesvector(g["rays"], ne_extent=1.5e-3, probing_direction=d,
                                              keep_current_plane=keep)
            assert none is None
            np.testing.assert_allclose(got, g[f"{d}_{int(keep)}"], rtol=1e-15)
        np.testing.assert_allclose(sp.back_propogate(g["rays"], 1.5e-3, d), g[f"bp_{d}"], rtol=1e-15)


def test_physics_matches_reference():
    for ne, Te, Z, om, kref in golden("kappa")["cases"]:
        assert physics.kappa_inv_brems(ne, Te, Z, om) == pytest.approx(kref, rel=1e-14)
        kq2, clw, ope2 = physics.kappa_factors(Te, Z, om)
        q = ne / physics.critical_density(om)
        cl = max(2.0, clw - 0.5 * np.log(max(ope2 * q, 1.0)))
        assert kq2 * q * q * cl * physics.C == pytest.approx(kref, rel=1e-12)
    om = physics.omega_of(532e-9)
    assert physics.critical_density(om) == pytest.approx(3.94e27, rel=1e-2)   # ~3.9e21 cm^-3 at 532 nm


def test_kolmogorov_field_statistics():
    n, L = 64, 5e-3
    ne = workloads.kolmogorov_box(n, L=L, seed=3).double()
    d = ne / 1e25 - 1.0
    assert abs(float(d.pow(2).mean().sqrt()) - 0.2) < 0.02          # 20 % RMS (before clipping)
    assert float(ne.min()) >= 0
    # radially averaged spectrum falls as k^-11/3 inside the band
    F = torch.fft.fftn(d).abs().pow(2)
    k = torch.fft.fftfreq(n) * n
    kk = torch.sqrt(k[:, None, None] ** 2 + k[None, :, None] ** 2 + k[None, None, :] ** 2)
    ks, ps = [], []
    for lo in range(2, 20):
        m = (kk >= lo) & (kk < lo + 1)
        ks.append(lo + 0.5)
        ps.append(float(F[m].mean()))
    slope = np.polyfit(np.log(ks), np.log(ps), 1)[0]
    assert abs(slope - (-11 / 3)) < 0.3
    a = workloads.kolmogorov_box(n, L=L, seed=3)
    b = workloads.kolmogorov_box(n, L=L, seed=3)
    assert torch.equal(a, b)


def test_beams_and_profiles():
    r = workloads.gaussian_beam(10000, waist=2e-3, seed=1, jitter=1e-3)
    assert r.shape == (6, 10000) and r.dtype == torch.float32
    assert abs(float(r[0].double().std()) - 1e-3) < 5e-5
    np.testing.assert_allclose(torch.linalg.norm(r[3:].double(), dim=0).numpy(), physics.C, rtol=1e-6)
    lat = workloads.lattice_beam(10, half_width=2e-3)
    assert lat.shape == (6, 100) and float(lat[0].max()) == pytest.approx(2e-3)
    s = workloads.sinusoid_slab(16)
    assert s.shape == (16, 16, 16) and float(s.max()) <= 1.1e24 * (1 + 1e-6)
    t = workloads.parabolic_trough(16)
    assert float(t.min()) >= 5e24 * (1 - 1e-6)


def test_serving_request_stream_statistics():
    from sloth_b200 import serving
    reqs = serving.request_stream(2000, rate=200.0, seed=0)
    t = np.array([r.t for r in reqs])
    assert np.all(np.diff(t) >= 0) and t[0] == 0.0
    assert abs(len(reqs) / t[-1] - 200.0) < 15.0                       # Poisson rate
    rays = np.array([r.rays for r in reqs])
    assert rays.min() >= 1e4 and rays.max() <= 4e6
    assert 1.6e5 < np.median(rays) < 2.5e5                             # lognormal median 2e5
    sizes = np.array([r.n for r in reqs])
    assert set(sizes) == {64, 128, 192, 256, 384}
    kinds = np.array([r.kind for r in reqs])
    assert 0.45 < (kinds == "kolmogorov").mean() < 0.55
    assert serving.request_stream(5, seed=1)[3] == serving.request_stream(5, seed=1)[3]
    keys = {serving.grid_key(r.kind, r.n, r.field_seed) for r in reqs}
    assert len(keys) <= 20
