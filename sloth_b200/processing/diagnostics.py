"""Ray-transfer-matrix diagnostics on the GPU: the API of the reference's
processing.diagnostics (src/processing/diagnostics.py), with the optics
chain and the detector histogram run by one kernel (K6, sloth_optics_*).

The solve methods of Shadowgraphy, Schlieren and Refractometry record their
chain of optics; Diagnostic.histogram runs the chain and bins the result in
one launch, without materialising the intermediate rays. ``rf`` after a
solve is produced on demand by the same kernel. The module-level optics
(lens, travel, the apertures and stops, knife_edge, lens_cutoff) take and
return numpy arrays like the reference's, and also run on the device.

Kept from the reference on purpose:
  * the chain arithmetic, bit for bit with numpy (fused multiply-add in
    travel, the NaN spread of the 4x4 products);
  * rect_aperture rejects rays only where BOTH |x| > Lx and |y| > Ly, as
    written at :94-104;
  * annular_stop returns the mask of rays between R1 and R2 (:83-92), as the
    reference does, instead of the rays;
  * histogram() without a solve bins ``rf`` as given (metres) against the
    detector size in mm, as the reference does.

Plotting (plot, plot_rays, plot_amplitude_diagnostics) is not part of this
library.
"""
from __future__ import annotations

import ctypes
from typing import List, Optional, Sequence, Tuple

import numpy as np
import torch

from .. import _capi as capi
from .. import runtime

TRAVEL = capi.SLOTH_OPTIC_TRAVEL
LENS = capi.SLOTH_OPTIC_LENS
CIRCULAR_APERTURE = capi.SLOTH_OPTIC_CIRCULAR_APERTURE
CIRCULAR_STOP = capi.SLOTH_OPTIC_CIRCULAR_STOP
RECT_APERTURE = capi.SLOTH_OPTIC_RECT_APERTURE
KNIFE_EDGE = capi.SLOTH_OPTIC_KNIFE_EDGE
ANNULAR_STOP = capi.SLOTH_OPTIC_ANNULAR_STOP

Op = Tuple[int, float, float, int]      # (kind, a, b, axis)


def _device_rays(r) -> torch.Tensor:
    dev = runtime.require_device()
    if isinstance(r, torch.Tensor):
        t = r
    else:
        t = torch.from_numpy(np.ascontiguousarray(r))
    if t.dtype not in (torch.float32, torch.float64):
        t = t.to(torch.float64)
    if t.device.type != "cuda":
        t = t.to(dev)
    return t.contiguous()


def run_optics(rays, ops: Sequence[Op] = (), *, weights=None, pos_scale: float = 1.0,
               prefilter: Optional[Tuple[float, float]] = None, ccd_half: Optional[Tuple[float, float]] = None,
               hist: Optional[Tuple[int, int, Tuple[float, float], Tuple[float, float]]] = None,
               want_rays: bool = False, want_kept: bool = False, out_hist: Optional[torch.Tensor] = None):
    """One K6 launch on (4, N) Jones vectors (numpy or torch; float32 or
    float64). Returns (rays_out (4, N) float64 tensor or None, kept (N,) bool
    tensor or None, histogram (ny, nx) float64 tensor or None).

    hist = (nx, ny, x_range, y_range); the histogram is added to `out_hist`
    when given, else to a new zeroed tensor."""
    r = _device_rays(rays)
    if r.dim() != 2 or r.shape[0] != 4:
        raise ValueError("rays must be (4, N)")
    n = int(r.shape[1])
    if len(ops) > capi.SLOTH_MAX_OPTICS:
        raise ValueError(f"at most {capi.SLOTH_MAX_OPTICS} optics per launch")
    arr = (capi.SlothOptic * max(len(ops), 1))()
    for k, (kind, a, b, axis) in enumerate(ops):
        arr[k].kind, arr[k].a, arr[k].b, arr[k].axis = int(kind), float(a), float(b), int(axis)
    d = capi.SlothDetectorParams()
    d.pos_scale = float(pos_scale)
    if prefilter is not None:
        d.prefilter, d.prefilter_L, d.prefilter_R = 1, float(prefilter[0]), float(prefilter[1])
    if ccd_half is not None:
        d.ccd_clip, d.ccd_half[0], d.ccd_half[1] = 1, float(ccd_half[0]), float(ccd_half[1])
    H = None
    if hist is not None:
        nx, ny, xr, yr = hist
        d.nx, d.ny = int(nx), int(ny)
        d.x_range[0], d.x_range[1] = float(xr[0]), float(xr[1])
        d.y_range[0], d.y_range[1] = float(yr[0]), float(yr[1])
        H = out_hist if out_hist is not None else torch.zeros((int(ny), int(nx)), dtype=torch.float64,
                                                              device=r.device)
    w = None
    if weights is not None:
        w = _device_rays(weights).to(r.dtype).contiguous()
        if w.numel() != n:
            raise ValueError("weights must have one entry per ray")
    rays_out = torch.empty((4, n), dtype=torch.float64, device=r.device) if want_rays else None
    kept = torch.empty(n, dtype=torch.uint8, device=r.device) if want_kept else None
    fn = capi.load().sloth_optics_f32 if r.dtype == torch.float32 else capi.load().sloth_optics_f64
    stream = torch.cuda.current_stream(r.device).cuda_stream
    capi.check(fn(capi.ptr(r), n, capi.ptr(w) if w is not None else None, arr, len(ops), ctypes.byref(d),
                  capi.ptr(H) if H is not None else None, capi.ptr(rays_out) if rays_out is not None else None,
                  capi.ptr(kept) if kept is not None else None, stream), "sloth_optics")
    return rays_out, (kept.bool() if kept is not None else None), H


# ---------------------------------------------------------------------------
# module-level optics (src/processing/diagnostics.py:16-150), numpy in/out
# ---------------------------------------------------------------------------
def m_to_mm(r):
    rr = np.copy(r)
    rr[0::2, :] *= 1e3
    return rr


def mm_to_m(r):
    rr = np.copy(r)
    rr[0::2, :] *= 1e-3
    return rr


def _apply(r, ops):
    out, _, _ = run_optics(r, ops, want_rays=True)
    return out.cpu().numpy()


def _reject_in_place(r, ops):
    out = _apply(r, ops)
    r[:, np.isnan(out[0]) & ~np.isnan(np.asarray(r[0], dtype=np.float64))] = np.nan
    return r


def lens(r, f1, f2):
    """Thin lens with focal lengths f1, f2 on the two axes."""
    return _apply(r, [(LENS, f1, f2, 0)])


def sym_lens(r, f):
    return lens(r, f, f)


def travel(r, d):
    """Free propagation over distance d."""
    return _apply(r, [(TRAVEL, d, 0.0, 0)])


def circular_aperture(r, R, E=None):
    """Rejects (sets to NaN, in place) rays outside radius R."""
    return _reject_in_place(r, [(CIRCULAR_APERTURE, R, 0.0, 0)])


def circular_stop(r, R):
    """Rejects (in place) rays inside radius R."""
    return _reject_in_place(r, [(CIRCULAR_STOP, R, 0.0, 0)])


def annular_stop(r, R1, R2):
    """Mask of the rays between R1 and R2 (the reference returns the mask)."""
    out = _apply(r, [(ANNULAR_STOP, R1, R2, 0)])
    return np.isnan(out[0]) & ~np.isnan(np.asarray(r[0], dtype=np.float64))


def rect_aperture(r, Lx, Ly):
    """Rejects (in place) rays with x^2 > Lx^2 and y^2 > Ly^2."""
    return _reject_in_place(r, [(RECT_APERTURE, Lx, Ly, 0)])


def knife_edge(r, offset, axis, direction):
    """Rejects (in place) rays beyond `offset` along 'x' or 'y' in the sense
    of `direction` (> 0: above, < 0: below)."""
    if axis not in ("x", "y"):
        raise ValueError("axis must be 'x' or 'y'")
    if direction == 0:
        raise ValueError("Direction must be <0 or >0")
    return _reject_in_place(r, [(KNIFE_EDGE, offset, 1.0 if direction > 0 else -1.0, 0 if axis == "x" else 2)])


def d2r(d):
    return d * np.pi / 180


def lens_cutoff(rf, *, L=400, R=25):
    """Rays whose straight line meets the next lens (distance L) within R."""
    _, kept, _ = run_optics(rf, [], prefilter=(L, R), want_kept=True)
    return np.asarray(rf)[:, kept.cpu().numpy()]


def clear_rays(self):
    """Drops the diagnostic's rays."""
    self._rf_in = None
    self._rf_custom = None
    self._rf_cache = None
    self._weights_dev = None


# ---------------------------------------------------------------------------
# Diagnostic classes (:176-380)
# ---------------------------------------------------------------------------
class Diagnostic:
    """Inheritable ray diagnostic; positions in mm after the solve."""

    def __init__(self, rf, *, weights=None, focal_plane=0, L=400, R=25, Lx=18, Ly=13.5, prefilter_input=False,
                 ccd_shape_m=None, verbose=True):
        self.focal_plane, self.L, self.R, self.Lx, self.Ly = focal_plane, L, R, Lx, Ly
        if ccd_shape_m is not None:
            self._ccd_half_x_mm = ccd_shape_m[0] * 1e3 / 2.0
            self._ccd_half_y_mm = ccd_shape_m[1] * 1e3 / 2.0
        else:
            self._ccd_half_x_mm = None
            self._ccd_half_y_mm = None
        if rf is None:
            raise ValueError("rf should not be None")
        assert rf.shape[0] == 4 or (len(rf.shape) == 3 and rf.shape[1] == 4), \
            "Incorrect format for rf, are you sure you passed the right variable?"
        if len(rf.shape) == 3:
            rf = rf[-1]
        t = _device_rays(rf)
        self.Np = int(t.shape[-1])
        w = None if weights is None else _device_rays(weights).to(torch.float64).reshape(-1)
        if prefilter_input:
            _, kept, _ = run_optics(t, [], prefilter=(self.L, self.R), want_kept=True)
            t = t[:, kept].contiguous()
            if w is not None:
                w = w[kept].contiguous()
        self.Np_inc = int(t.shape[-1])
        if verbose:
            if self.Np == self.Np_inc:
                print("\nAll rays retained at diagnostic input.")
            else:
                print(f"\n{self.Np} rays received, {self.Np_inc} retained after optional prefilter.")
                print(f" --> {round((1 - self.Np_inc / self.Np) * 100, 3)} % filtered before diagnostic solve.")
        self._rf_in = t                   # device, metres, caller's precision
        self._weights_dev = w
        self.weights = None if w is None else w.cpu().numpy()
        self._ops: Optional[List[Op]] = None
        self._rf_custom = None
        self._rf_cache = None

    # rays -------------------------------------------------------------------
    @property
    def r0(self):
        if self._rf_in is None:
            return None
        return m_to_mm(self._rf_in.cpu().numpy())

    @property
    def rf(self):
        if self._rf_custom is not None:
            return self._rf_custom
        if self._rf_in is None:
            return None
        if self._ops is None:
            return self._rf_in.cpu().numpy()
        if self._rf_cache is None:
            out, _, _ = run_optics(self._rf_in, self._ops, pos_scale=1e3, want_rays=True)
            self._rf_cache = out.cpu().numpy()
        return self._rf_cache

    @rf.setter
    def rf(self, value):
        self._rf_custom = value
        self._rf_cache = None

    def _solve(self, ops: List[Op]):
        self._ops = list(ops)
        self._rf_custom = None
        self._rf_cache = None

    # detector ---------------------------------------------------------------
    def histogram(self, *, bin_scale=1, pix_x=3448, pix_y=2574, clear_mem=False, plain_plot=False,
                  extra_info=True):
        """Bin the rays into a pix_x/bin_scale x pix_y/bin_scale image over the
        detector (Lx x Ly mm): self.H (transposed, as the reference),
        self.xedges, self.yedges."""
        nx = int(np.floor(pix_x / bin_scale))
        ny = int(np.floor(pix_y / bin_scale))
        xr, yr = (-self.Lx / 2, self.Lx / 2), (-self.Ly / 2, self.Ly / 2)
        ccd = None if self._ccd_half_x_mm is None else (self._ccd_half_x_mm, self._ccd_half_y_mm)
        if plain_plot:
            src, ops, scale = self._rf_in, [], 1e3
        elif self._rf_custom is not None:
            src, ops, scale = self._rf_custom, [], 1.0
        elif self._ops is None:
            src, ops, scale = self._rf_in, [], 1.0
        else:
            src, ops, scale = self._rf_in, self._ops, 1e3
        _, _, H = run_optics(src, ops, weights=self._weights_dev, pos_scale=scale, ccd_half=ccd,
                             hist=(nx, ny, xr, yr))
        self.H = H.cpu().numpy()
        self.xedges = np.linspace(xr[0], xr[1], nx + 1)
        self.yedges = np.linspace(yr[0], yr[1], ny + 1)
        if clear_mem:
            clear_rays(self)

    def plot(self, *a, **k):
        raise NotImplementedError("plotting is not part of sloth_b200; plot self.H with matplotlib")

    def plot_rays(self, *a, **k):
        raise NotImplementedError("plotting is not part of sloth_b200")


class Shadowgraphy(Diagnostic):
    """Shadowgraphy: single-lens (M ~ 2) and two-lens (M = 1) imaging
    (src/processing/diagnostics.py:270-306)."""

    def single_lens_custom_solve(self, f=200, obj_dist=400, img_dist=400):
        self._solve([(TRAVEL, obj_dist - self.focal_plane, 0, 0), (CIRCULAR_APERTURE, self.R, 0, 0),
                     (LENS, f, f, 0), (TRAVEL, img_dist, 0, 0)])

    def single_lens_solve(self):
        L = self.L
        self._solve([(TRAVEL, 3 * L / 4 - self.focal_plane, 0, 0), (CIRCULAR_APERTURE, self.R, 0, 0),
                     (LENS, L / 2, L / 2, 0), (TRAVEL, 3 * L / 2, 0, 0)])

    def two_lens_solve(self):
        L = self.L
        self._solve([(TRAVEL, L - self.focal_plane, 0, 0), (CIRCULAR_APERTURE, self.R, 0, 0),
                     (LENS, L / 2, L / 2, 0), (TRAVEL, L * 2, 0, 0), (CIRCULAR_APERTURE, self.R, 0, 0),
                     (LENS, L / 2, L / 2, 0), (TRAVEL, L, 0, 0)])


class Schlieren(Diagnostic):
    """Dark- and light-field schlieren: a two-lens telescope with a stop or
    aperture of radius R at the focal point (:308-350)."""

    def DF_solve(self, R=1):
        L = self.L
        self._solve([(TRAVEL, L - self.focal_plane, 0, 0), (CIRCULAR_APERTURE, self.R, 0, 0), (LENS, L, L, 0),
                     (TRAVEL, L, 0, 0), (CIRCULAR_STOP, R, 0, 0), (TRAVEL, L, 0, 0),
                     (CIRCULAR_APERTURE, self.R, 0, 0), (LENS, L, L, 0), (TRAVEL, L, 0, 0)])

    def LF_solve(self, R=1):
        L = self.L
        self._solve([(TRAVEL, L - self.focal_plane, 0, 0), (CIRCULAR_APERTURE, self.R, 0, 0), (LENS, L, L, 0),
                     (TRAVEL, L, 0, 0), (CIRCULAR_APERTURE, R, 0, 0), (TRAVEL, L, 0, 0),
                     (CIRCULAR_APERTURE, self.R, 0, 0), (LENS, L, L, 0), (TRAVEL, L, 0, 0)])


class Refractometry(Diagnostic):
    """Imaging refractometer: spherical then hybrid lens (:352-380)."""

    def incoherent_custom_solve(self, f1=200, f3=200, img_f1_dist=600, img_dist=400):
        self._solve([(TRAVEL, 2 * f1 - self.focal_plane, 0, 0), (CIRCULAR_APERTURE, self.R, 0, 0),
                     (LENS, f1, f1, 0), (TRAVEL, img_f1_dist, 0, 0), (RECT_APERTURE, 15, 30, 0),
                     (CIRCULAR_APERTURE, self.R, 0, 0), (LENS, (2 * f3) / 3, f1, 0), (TRAVEL, img_dist, 0, 0)])

    def incoherent_solve(self):
        L = self.L
        self._solve([(TRAVEL, 3 * L / 4 - self.focal_plane, 0, 0), (CIRCULAR_APERTURE, self.R, 0, 0),
                     (LENS, L / 2, L / 2, 0), (TRAVEL, 3 * L / 2, 0, 0), (RECT_APERTURE, 15, 30, 0),
                     (CIRCULAR_APERTURE, self.R, 0, 0), (LENS, L / 3, L / 2, 0), (TRAVEL, L, 0, 0)])
