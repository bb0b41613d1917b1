"""Jones-vector projection of ray states (src/shared/propagation.py:4-134).

The tracers fuse this projection into their epilogue; these host versions
keep the reference's functions available for arrays already on the host.
"""
from __future__ import annotations

import numpy as np


def _axes(probing_direction):
    if probing_direction == 'x':
        return 0, 1, 2
    if probing_direction == 'y':
        return 1, 0, 2
    if probing_direction == 'z':
        return 2, 0, 1
    return None


def ray_to_Jonesvector(rays, *, ne_extent=None, probing_direction='z', keep_current_plane=False):
    """(4, N) rows (pos1, angle1, pos2, angle2) of (6, N) rays; with
    keep_current_plane=False the rays are first moved along v onto the plane
    probing_axis = ne_extent (:4-90). Returns (ray_p, None)."""
    if ne_extent is None and not keep_current_plane:
        print("\nne_extent is only not required if keep_current_plane is set to True, setting "
              "keep_current_plane = True for you.")
        keep_current_plane = True
    rays = np.asarray(rays)
    out = np.zeros((4, rays.shape[1]), dtype=np.result_type(rays.dtype, np.float32))
    ax = _axes(probing_direction)
    if ax is None:
        print("\nIncorrect probing direction. Use: x, y or z.")
        return out, None
    a, t1, t2 = ax
    if keep_current_plane:
        out[0], out[2] = rays[t1], rays[t2]
    else:
        t_bp = (rays[a] - ne_extent) / rays[3 + a]
        out[0] = rays[t1] - rays[3 + t1] * t_bp
        out[2] = rays[t2] - rays[3 + t2] * t_bp
    out[1] = np.arctan(rays[3 + t1] / rays[3 + a])
    out[3] = np.arctan(rays[3 + t2] / rays[3 + a])
    return out, None


def back_propogate(rays, ne_extent, probing_direction):
    """Rays moved along v onto the plane probing_axis = ne_extent (:92-134)."""
    rays = np.array(rays, copy=True)
    ax = _axes(probing_direction)
    if ax is None:
        print("\nIncorrect probing direction. Use: x, y or z.")
        return rays
    a, t1, t2 = ax
    t_bp = (rays[a] - ne_extent) / rays[3 + a]
    rays[t1] = rays[t1] - rays[3 + t1] * t_bp
    rays[t2] = rays[t2] - rays[3 + t2] * t_bp
    rays[a] = ne_extent
    return rays


back_propagate = back_propogate
