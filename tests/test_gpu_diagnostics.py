"""Ray-transfer-matrix diagnostics on the GPU (K6, sloth_optics_*): the
Shadowgraphy / Schlieren / Refractometry mirrors and the module-level optics
against the reference's own outputs (bit for bit), the kernel against the
numpy oracle on 1e6 rays, error codes, and a trace feeding a diagnostic on
the device."""
import ctypes

import numpy as np
import pytest
import torch

from conftest import golden
from oracle import diagnostics_np as dn
from sloth_b200 import _capi
from sloth_b200.processing import diagnostics as dg

pytestmark = pytest.mark.gpu

CASES = {
    "shadow_single": (dg.Shadowgraphy, "single_lens_solve", {}, dict(bin_scale=16), {}, True),
    "shadow_two": (dg.Shadowgraphy, "two_lens_solve", dict(focal_plane=1.0), dict(bin_scale=8), {}, False),
    "shadow_custom": (dg.Shadowgraphy, "single_lens_custom_solve", dict(prefilter_input=True,
                                                                        ccd_shape_m=(10e-3, 8e-3)),
                      dict(bin_scale=12), dict(f=150, obj_dist=300, img_dist=600), True),
    "schlieren_df": (dg.Schlieren, "DF_solve", {}, dict(bin_scale=16), dict(R=1.0), True),
    "schlieren_lf": (dg.Schlieren, "LF_solve", {}, dict(bin_scale=16), dict(R=1.0), True),
    "refract": (dg.Refractometry, "incoherent_solve", {}, dict(bin_scale=16), {}, True),
    "refract_custom": (dg.Refractometry, "incoherent_custom_solve", {}, dict(bin_scale=16),
                       dict(f1=150, f3=250, img_f1_dist=500, img_dist=350), True),
    "plain": (dg.Shadowgraphy, None, {}, dict(bin_scale=16, plain_plot=True), {}, True),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_diagnostics_match_reference(name):
    g = golden("diagnostics")
    cls, solve, init_kw, hist_kw, solve_kw, use_w = CASES[name]
    d = cls(g["rf"].copy(), weights=g["weights"].copy() if use_w else None, L=400, R=25, Lx=18, Ly=13.5,
            verbose=False, **init_kw)
    if solve:
        getattr(d, solve)(**solve_kw)
    d.histogram(**hist_kw)
    np.testing.assert_array_equal(d.H, g[f"{name}_H"])
    np.testing.assert_array_equal(d.xedges, g[f"{name}_xedges"])
    np.testing.assert_array_equal(d.yedges, g[f"{name}_yedges"])
    np.testing.assert_array_equal(np.asarray(d.rf, dtype=np.float64), g[f"{name}_rf"])


def test_module_optics_match_reference():
    g = golden("diagnostics")
    r = g["op_in"]
    np.testing.assert_array_equal(dg.travel(r, 123.0), g["op_travel"])
    np.testing.assert_array_equal(dg.lens(r, 80.0, -120.0), g["op_lens"])
    np.testing.assert_array_equal(dg.circular_aperture(r.copy(), 2.5), g["op_circ_ap"])
    np.testing.assert_array_equal(dg.circular_stop(r.copy(), 1.5), g["op_circ_stop"])
    np.testing.assert_array_equal(dg.rect_aperture(r.copy(), 2.0, 1.0), g["op_rect_ap"])
    np.testing.assert_array_equal(dg.annular_stop(r.copy(), 1.0, 2.5), g["op_annular_mask"])
    np.testing.assert_array_equal(dg.knife_edge(r.copy(), 0.5, "x", 1), g["op_knife_x_pos"])
    np.testing.assert_array_equal(dg.knife_edge(r.copy(), -0.25, "y", -1), g["op_knife_y_neg"])
    np.testing.assert_array_equal(dg.lens_cutoff(r.copy(), L=400, R=3), g["op_lens_cutoff"])
    with pytest.raises(ValueError):
        dg.knife_edge(r.copy(), 0.0, "x", 0)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_kernel_matches_oracle_on_1e6_rays(dtype):
    rng = np.random.default_rng(5)
    N = 1_000_000
    rf = np.stack([rng.normal(0, 2e-3, N), rng.normal(0, 6e-3, N), rng.normal(0, 2e-3, N),
                   rng.normal(0, 6e-3, N)]).astype(dtype)
    rf[:, rng.integers(0, N, 50)] = np.nan
    w = rng.uniform(0.2, 1.0, N).astype(dtype)
    ops = dn.schlieren_df(400, 25, 0.5, stop=0.8) + [(dn.KNIFE_EDGE, 1.5, 1.0, 0), (dn.ANNULAR_STOP, 2.0, 2.5, 0)]
    out, kept, H = dg.run_optics(rf, ops, weights=w, pos_scale=1e3, prefilter=(400, 25), ccd_half=(8.0, 6.0),
                                 hist=(431, 321, (-9.0, 9.0), (-6.75, 6.75)), want_rays=True, want_kept=True)
    m = dn.prefilter_mask(rf, 400, 25)
    np.testing.assert_array_equal(kept.cpu().numpy(), m)
    ref = dn.apply_optics(dn.m_to_mm(rf[:, m]), ops)
    np.testing.assert_array_equal(out.cpu().numpy()[:, m], ref)
    assert np.isnan(out.cpu().numpy()[:, ~m]).all()
    Hr, _, _ = dn.histogram(ref, w[m], pix_x=431, pix_y=321, bin_scale=1, Lx=18, Ly=13.5, ccd_half=(8.0, 6.0))
    np.testing.assert_allclose(H.cpu().numpy(), Hr, rtol=1e-12, atol=0)
    _, _, Hc = dg.run_optics(rf, ops, pos_scale=1e3, prefilter=(400, 25), ccd_half=(8.0, 6.0),
                             hist=(431, 321, (-9.0, 9.0), (-6.75, 6.75)))
    Hcr, _, _ = dn.histogram(ref, None, pix_x=431, pix_y=321, bin_scale=1, Lx=18, Ly=13.5, ccd_half=(8.0, 6.0))
    np.testing.assert_array_equal(Hc.cpu().numpy(), Hcr)
    assert Hcr.sum() > 1000


def test_values_on_bin_edges_follow_numpy():
    # points exactly on every edge, on the upper range end, and just outside
    edges = np.linspace(-9.0, 9.0, 37)
    x = np.concatenate([edges, [9.0, -9.0, np.nextafter(9.0, 10), np.nextafter(-9.0, -10)]])
    rf = np.stack([x, np.zeros_like(x), np.zeros_like(x), np.zeros_like(x)])
    _, _, H = dg.run_optics(rf, [], hist=(36, 1, (-9.0, 9.0), (-1.0, 1.0)))
    ref, _, _ = np.histogram2d(x, np.zeros_like(x), bins=[36, 1], range=[[-9.0, 9.0], [-1.0, 1.0]])
    np.testing.assert_array_equal(H.cpu().numpy(), ref.T)


def test_error_codes():
    lib = _capi.load()
    r = torch.zeros((4, 8), dtype=torch.float64, device="cuda")
    d = _capi.SlothDetectorParams()
    d.pos_scale = 1.0
    ops = (_capi.SlothOptic * 40)()

    def call(n_ops, dd=d, hist=None):
        return lib.sloth_optics_f64(_capi.ptr(r), 8, None, ops, n_ops, ctypes.byref(dd), hist, None, None, None)

    ops[0].kind = _capi.SLOTH_OPTIC_TRAVEL
    assert call(1) == _capi.SLOTH_OK
    assert call(33) == _capi.SLOTH_ERR_INVALID_ARGUMENT
    ops[0].kind = 99
    assert call(1) == _capi.SLOTH_ERR_INVALID_ARGUMENT
    ops[0].kind, ops[0].a, ops[0].b = _capi.SLOTH_OPTIC_LENS, 0.0, 1.0
    assert call(1) == _capi.SLOTH_ERR_INVALID_ARGUMENT
    ops[0].kind, ops[0].axis, ops[0].b = _capi.SLOTH_OPTIC_KNIFE_EDGE, 1, 1.0
    assert call(1) == _capi.SLOTH_ERR_INVALID_ARGUMENT
    h = torch.zeros(4, dtype=torch.float64, device="cuda")
    d2 = _capi.SlothDetectorParams()
    d2.pos_scale, d2.nx, d2.ny = 1.0, 2, 2
    d2.x_range[0], d2.x_range[1], d2.y_range[0], d2.y_range[1] = 1.0, 1.0, 0.0, 1.0
    assert call(0, d2, _capi.ptr(h)) == _capi.SLOTH_ERR_INVALID_ARGUMENT
    d2.x_range[1] = 2.0
    assert call(0, d2, _capi.ptr(h)) == _capi.SLOTH_OK
    d2.pos_scale = 0.0
    assert call(0, d2, _capi.ptr(h)) == _capi.SLOTH_ERR_INVALID_ARGUMENT
    torch.cuda.synchronize()


def test_trace_to_diagnostic_on_device():
    """solve()'s rays and transmission feed a Shadowgraphy histogram; the
    device-resident path gives the reference's numpy histogram."""
    from sloth_b200 import runtime, workloads
    from sloth_b200.core import physics
    L, n = 5e-3, 64
    h = L / (n - 1)
    ne = workloads.kolmogorov_box(n, L=L, mean=1e25, rms=0.2, seed=3)
    rays = workloads.gaussian_beam(200_000, waist=1.5e-3, L=L, seed=4, device="cuda")
    g = runtime.pack_grid(ne, (-L / 2,) * 3, (h,) * 3, physics.omega_of(532e-9))
    sched = runtime.schedule_times([np.sqrt(8.0) * L], (h, h, h))
    out = runtime.trace(g, rays, sched, project=True, plane=L / 2, inv_brems=True, Te=20.0, Z=1.0)
    jv, amp = out["jones"][-1], out["amp"][-1]
    d = dg.Shadowgraphy(jv, weights=amp, L=400, R=25, Lx=18, Ly=13.5, verbose=False)
    d.single_lens_solve()
    d.histogram(bin_scale=4)
    r = dn.apply_optics(dn.m_to_mm(jv.cpu().numpy()), dn.shadow_single(400, 25, 0.0))
    Hr, _, _ = dn.histogram(r, amp.cpu().numpy(), pix_x=3448, pix_y=2574, bin_scale=4, Lx=18, Ly=13.5)
    np.testing.assert_allclose(d.H, Hr, rtol=1e-12, atol=0)
    assert d.H.sum() > 0.5 * 200_000 * float(amp.min())
