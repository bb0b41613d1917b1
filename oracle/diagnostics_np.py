"""Test infrastructure only: a numpy restatement of the reference's
ray-transfer-matrix diagnostics (src/processing/diagnostics.py), written
against the op list of the device kernel, the thing it checks:
(kind, a, b, axis) with the kinds of include/sloth_b200.h SLOTH_OPTIC_*.
It is pinned to the reference's own outputs in tests/golden/diagnostics.npz.

Reference semantics restated:
  * travel and lens (:28-61) are 4x4 matrix products (np.matmul, whose
    BLAS accumulates each row with fused multiply-adds in column order):
    travel x' = fma(d, theta, x), one rounding; lens theta' =
    round(round((-1/f)*x) + theta); a NaN anywhere in a ray makes all four
    rows NaN;
  * apertures and stops (:63-123) set the whole ray to NaN where their
    condition holds; NaN rays never satisfy a condition;
  * m_to_mm (:16-20) multiplies rows 0 and 2 in the array's own dtype;
  * the lens-cutoff prefilter (:223-231) and the CCD clip (:249-255);
  * Diagnostic.histogram (:238-262): numpy.histogram2d over
    [-Lx/2, Lx/2] x [-Ly/2, Ly/2], floor(pix/bin_scale) bins, transposed.
"""
from __future__ import annotations

import numpy as np

TRAVEL, LENS, CIRCULAR_APERTURE, CIRCULAR_STOP, RECT_APERTURE, KNIFE_EDGE, ANNULAR_STOP = range(1, 8)


def _two_prod(a, b):
    """p + e == a*b exactly (Veltkamp splitting)."""
    p = a * b
    sp = 134217729.0
    ah = a * sp
    ah = ah - (ah - a)
    al = a - ah
    bh = b * sp
    bh = bh - (bh - b)
    bl = b - bh
    e = ((ah * bh - p) + ah * bl + al * bh) + al * bl
    return p, e


def fma(a, b, c):
    """a*b + c with one rounding (error-free transformations; exact except in
    double-rounding corner cases that these tests never meet)."""
    p, e = _two_prod(np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64))
    s = p + c
    bb = s - p
    t = (p - (s - bb)) + (c - bb)
    return s + (t + e)


def apply_optics(r, ops):
    """Apply the op list to (4, N) float64 rays (a copy is returned)."""
    r = np.array(r, dtype=np.float64, copy=True)
    for kind, a, b, axis in ops:
        if kind in (TRAVEL, LENS):
            bad = np.isnan(r).any(axis=0)
            if kind == TRAVEL:
                with np.errstate(invalid="ignore"):
                    r[0] = fma(a, r[1], r[0])
                    r[2] = fma(a, r[3], r[2])
            else:
                r[1] = (-1.0 / a) * r[0] + r[1]
                r[3] = (-1.0 / b) * r[2] + r[3]
            r[:, bad] = np.nan
            continue
        r2 = r[0] ** 2 + r[2] ** 2
        with np.errstate(invalid="ignore"):
            if kind == CIRCULAR_APERTURE:
                f = r2 > a ** 2
            elif kind == CIRCULAR_STOP:
                f = r2 < a ** 2
            elif kind == RECT_APERTURE:
                f = (r[0] ** 2 > a ** 2) & (r[2] ** 2 > b ** 2)
            elif kind == KNIFE_EDGE:
                v = r[axis]
                f = (v > a) if b > 0 else (v < a)
            elif kind == ANNULAR_STOP:
                f = (r2 > a ** 2) & (r2 < b ** 2)
            else:
                raise ValueError(kind)
        r[:, f] = np.nan
    return r


def prefilter_mask(rf, L, R):
    xp = L * np.tan(rf[1]) + rf[0]
    yp = L * np.tan(rf[3]) + rf[2]
    with np.errstate(invalid="ignore"):
        return np.sqrt(xp ** 2 + yp ** 2) <= R


def m_to_mm(rf):
    r = np.copy(rf)
    r[0::2, :] *= 1e3
    return r


def histogram(r, weights, *, pix_x, pix_y, bin_scale, Lx, Ly, ccd_half=None):
    mask = ~np.isnan(r[0]) & ~np.isnan(r[2])
    if ccd_half is not None:
        mask &= (np.abs(r[0]) <= ccd_half[0]) & (np.abs(r[2]) <= ccd_half[1])
    w = None if weights is None else np.asarray(weights, dtype=np.float64)[mask]
    H, xe, ye = np.histogram2d(r[0, mask], r[2, mask], bins=[int(pix_x // bin_scale), int(pix_y // bin_scale)],
                               range=[[-Lx / 2, Lx / 2], [-Ly / 2, Ly / 2]], weights=w)
    return H.T, xe, ye


# The reference's solve methods as op lists (src/processing/diagnostics.py:286-380).
def shadow_single(L, R, fp):
    return [(TRAVEL, 3 * L / 4 - fp, 0, 0), (CIRCULAR_APERTURE, R, 0, 0), (LENS, L / 2, L / 2, 0),
            (TRAVEL, 3 * L / 2, 0, 0)]


def shadow_custom(L, R, fp, f=200, obj_dist=400, img_dist=400):
    return [(TRAVEL, obj_dist - fp, 0, 0), (CIRCULAR_APERTURE, R, 0, 0), (LENS, f, f, 0), (TRAVEL, img_dist, 0, 0)]


def shadow_two(L, R, fp):
    return [(TRAVEL, L - fp, 0, 0), (CIRCULAR_APERTURE, R, 0, 0), (LENS, L / 2, L / 2, 0), (TRAVEL, 2 * L, 0, 0),
            (CIRCULAR_APERTURE, R, 0, 0), (LENS, L / 2, L / 2, 0), (TRAVEL, L, 0, 0)]


def schlieren_df(L, R, fp, stop=1.0):
    return [(TRAVEL, L - fp, 0, 0), (CIRCULAR_APERTURE, R, 0, 0), (LENS, L, L, 0), (TRAVEL, L, 0, 0),
            (CIRCULAR_STOP, stop, 0, 0), (TRAVEL, L, 0, 0), (CIRCULAR_APERTURE, R, 0, 0), (LENS, L, L, 0),
            (TRAVEL, L, 0, 0)]


def schlieren_lf(L, R, fp, stop=1.0):
    return [(TRAVEL, L - fp, 0, 0), (CIRCULAR_APERTURE, R, 0, 0), (LENS, L, L, 0), (TRAVEL, L, 0, 0),
            (CIRCULAR_APERTURE, stop, 0, 0), (TRAVEL, L, 0, 0), (CIRCULAR_APERTURE, R, 0, 0), (LENS, L, L, 0),
            (TRAVEL, L, 0, 0)]


def refract(L, R, fp):
    return [(TRAVEL, 3 * L / 4 - fp, 0, 0), (CIRCULAR_APERTURE, R, 0, 0), (LENS, L / 2, L / 2, 0),
            (TRAVEL, 3 * L / 2, 0, 0), (RECT_APERTURE, 15, 30, 0), (CIRCULAR_APERTURE, R, 0, 0),
            (LENS, L / 3, L / 2, 0), (TRAVEL, L, 0, 0)]


def refract_custom(L, R, fp, f1=200, f3=200, img_f1_dist=600, img_dist=400):
    return [(TRAVEL, 2 * f1 - fp, 0, 0), (CIRCULAR_APERTURE, R, 0, 0), (LENS, f1, f1, 0),
            (TRAVEL, img_f1_dist, 0, 0), (RECT_APERTURE, 15, 30, 0), (CIRCULAR_APERTURE, R, 0, 0),
            (LENS, (2 * f3) / 3, f1, 0), (TRAVEL, img_dist, 0, 0)]
