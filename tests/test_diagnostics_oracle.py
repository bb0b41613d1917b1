"""CPU checks of the diagnostics oracle (oracle/diagnostics_np.py) against the
reference's own Shadowgraphy / Schlieren / Refractometry solves, histograms
and module-level optics (tests/golden/diagnostics.npz)."""
import numpy as np
import pytest

from conftest import golden
from oracle import diagnostics_np as dn

G = dict(L=400, R=25, fp=0.0)
CASES = {
    # name: (ops, bin_scale, focal_plane, weights, prefilter, ccd_half)
    "shadow_single": (dn.shadow_single(400, 25, 0.0), 16, True, False, None),
    "shadow_two": (dn.shadow_two(400, 25, 1.0), 8, False, False, None),
    "shadow_custom": (dn.shadow_custom(400, 25, 0.0, f=150, obj_dist=300, img_dist=600), 12, True, True, (5.0, 4.0)),
    "schlieren_df": (dn.schlieren_df(400, 25, 0.0, stop=1.0), 16, True, False, None),
    "schlieren_lf": (dn.schlieren_lf(400, 25, 0.0, stop=1.0), 16, True, False, None),
    "refract": (dn.refract(400, 25, 0.0), 16, True, False, None),
    "refract_custom": (dn.refract_custom(400, 25, 0.0, f1=150, f3=250, img_f1_dist=500, img_dist=350), 16, True,
                       False, None),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_solves_and_histograms_match_reference(name):
    g = golden("diagnostics")
    ops, bs, use_w, pre, ccd = CASES[name]
    rf, w = g["rf"], g["weights"]
    if pre:
        m = dn.prefilter_mask(rf, 400, 25)
        rf, w = rf[:, m], w[m]
    r = dn.apply_optics(dn.m_to_mm(rf), ops)
    np.testing.assert_array_equal(r, g[f"{name}_rf"])
    H, xe, ye = dn.histogram(r, w if use_w else None, pix_x=3448, pix_y=2574, bin_scale=bs, Lx=18, Ly=13.5,
                             ccd_half=ccd)
    np.testing.assert_array_equal(H, g[f"{name}_H"])
    np.testing.assert_array_equal(xe, g[f"{name}_xedges"])
    np.testing.assert_array_equal(ye, g[f"{name}_yedges"])


def test_plain_histogram_and_module_optics_match_reference():
    g = golden("diagnostics")
    H, _, _ = dn.histogram(dn.m_to_mm(g["rf"]), g["weights"], pix_x=3448, pix_y=2574, bin_scale=16, Lx=18, Ly=13.5)
    np.testing.assert_array_equal(H, g["plain_H"])
    r = g["op_in"]
    T = dn
    for key, ops in (("op_travel", [(T.TRAVEL, 123.0, 0, 0)]), ("op_lens", [(T.LENS, 80.0, -120.0, 0)]),
                     ("op_circ_ap", [(T.CIRCULAR_APERTURE, 2.5, 0, 0)]),
                     ("op_circ_stop", [(T.CIRCULAR_STOP, 1.5, 0, 0)]),
                     ("op_rect_ap", [(T.RECT_APERTURE, 2.0, 1.0, 0)]),
                     ("op_knife_x_pos", [(T.KNIFE_EDGE, 0.5, 1, 0)]),
                     ("op_knife_y_neg", [(T.KNIFE_EDGE, -0.25, -1, 2)])):
        np.testing.assert_array_equal(dn.apply_optics(r, ops), g[key], err_msg=key)
    out = dn.apply_optics(r, [(T.ANNULAR_STOP, 1.0, 2.5, 0)])
    np.testing.assert_array_equal(np.isnan(out[0]) & ~np.isnan(r[0]), g["op_annular_mask"])
    m = dn.prefilter_mask(r, 400, 3)
    np.testing.assert_array_equal(r[:, m], g["op_lens_cutoff"])
