"""Beam: initial rays (6, N) = (x, y, z, vx, vy, vz) of a probing beam.

Mirrors core.beam.Beam of the reference (src/core/beam.py:6-371): same
constructor, the same single numpy RandomState stream drawn in the same order
(seed 42 when ``seeded``), rays starting on the plane probing_axis =
-ne_extent at speed c. The trigonometry is evaluated in float64 and the rays
are returned as float32 like the reference's default (x32) jnp arrays, so
seeded beams agree with the reference to float32 rounding.

Differences, each a defect of the reference:
* 'linear' raises UnboundLocalError in the reference (:238-254 never bind u,
  phi before the deletes at :338-341); here it returns the line beam that
  code describes.
* 'even' never writes s0 and fails on a float range() (:255-272); here it
  raises NotImplementedError.
* unknown beam types print a message and then fail on `del t` (:335-338);
  here they raise ValueError with that message.

Keyword-only extra: ``device`` (e.g. 'cuda') generates the rays on the GPU
(sloth_beam_f32) into a CUDA tensor ``s0``, for beams too large to draw on
the host. Those rays follow the same distributions and placement, but their
random numbers come from a counter-based hash of (seed, ray index), not from
numpy's RandomState, so a seeded device beam is reproducible but is not the
reference's seeded beam.
"""
from __future__ import annotations

import ctypes
import secrets

import numpy as np
from scipy.constants import c

_VALID_TYPES = (int, float, np.integer, np.floating)


class Beam:
    def __init__(self, Np, beam_size, divergence, ne_extent, *, probing_direction='z', beam_type='circular',
                 seeded=False, device=None):
        self.Np = np.int64(Np)
        self.beam_size = beam_size
        self.divergence = divergence
        self.ne_extent = ne_extent
        self.probing_direction = probing_direction
        self.beam_type = beam_type
        self.seed = 42 if seeded else None
        if device is not None:
            self._init_beam_device(-self.ne_extent, device)
        else:
            Beam.init_beam(self, -self.ne_extent, self.seed)

    def _init_beam_device(self, ne_extent, device):
        import torch
        from .. import _capi as capi
        from .. import runtime
        bt = self.beam_type
        kinds = {'circular': capi.SLOTH_BEAM_CIRCULAR, 'square': capi.SLOTH_BEAM_SQUARE,
                 'rectangular': capi.SLOTH_BEAM_RECTANGULAR, 'rect_trackers': capi.SLOTH_BEAM_RECTANGULAR,
                 'linear': capi.SLOTH_BEAM_LINEAR}
        if bt == 'even':
            raise NotImplementedError("beam_type 'even' produces no rays in the reference (src/core/beam.py:255-272)")
        if bt not in kinds:
            raise ValueError("\nself.beam_type unrecognised! Accepted args: circular, square, rectangular, linear, "
                             "even, rect_trackers.")
        if bt in ('rectangular', 'rect_trackers'):
            assert len(self.beam_size) == 2, ("\nERROR: Must pass a list of length 2 to initialise a rectangular beam,"
                                              + str(len(self.beam_size)) + "item was passed.")
            size = (float(self.beam_size[0]), float(self.beam_size[1]))
        else:
            assert isinstance(self.beam_size, _VALID_TYPES), \
                "\nReceived beam_size of shape" + str(np.shape(self.beam_size)) + "expected a float."
            size = (float(self.beam_size), 0.0)
        dev = runtime.require_device(device)
        p = capi.SlothBeamParams()
        p.beam_type = kinds[bt]
        p.probing_axis = ['x', 'y', 'z'].index(self.probing_direction)
        p.size[0], p.size[1] = size
        p.divergence = float(self.divergence)
        p.ne_extent = float(ne_extent)
        p.seed = self.seed if self.seed is not None else secrets.randbits(64)
        p.first_id = 0
        n = int(self.Np)
        s0 = torch.empty((6, n), dtype=torch.float32, device=dev)
        capi.check(capi.load().sloth_beam_f32(ctypes.byref(p), n, capi.ptr(s0),
                                              torch.cuda.current_stream(dev).cuda_stream), "sloth_beam_f32")
        self.s0 = s0

    def init_beam(self, ne_extent, seed):
        rng = np.random.RandomState(seed)
        Np = int(self.Np)
        s0 = np.zeros((6, Np), dtype=np.float64)
        d = self.probing_direction
        bt = self.beam_type

        def velocity(chi, phi):
            # (along, transverse-1, transverse-2) components as in :115-145
            if d == 'x':
                s0[3], s0[4], s0[5] = c * np.cos(chi), c * np.sin(chi) * np.cos(phi), c * np.sin(chi) * np.sin(phi)
            elif d == 'z':
                s0[3], s0[4], s0[5] = c * np.sin(chi) * np.cos(phi), c * np.sin(chi) * np.sin(phi), c * np.cos(chi)
            else:
                s0[4], s0[3], s0[5] = c * np.cos(chi), c * np.sin(chi) * np.cos(phi), c * np.sin(chi) * np.sin(phi)

        def position(a, b):
            # (a, b) are the in-plane coordinates; the probing coordinate is ne_extent
            if d == 'x':
                s0[0], s0[1], s0[2] = ne_extent, a, b
            elif d == 'z':
                s0[0], s0[1], s0[2] = a, b, ne_extent
            else:
                s0[0], s0[1], s0[2] = a, ne_extent, b

        if bt == 'circular':
            assert isinstance(self.beam_size, _VALID_TYPES), \
                "\nReceived beam_size of shape" + str(np.shape(self.beam_size)) + "expected a float."
            t = 2 * np.pi * rng.rand(Np)
            u = rng.power(2, Np)
            phi = np.pi * rng.rand(Np)
            chi = self.divergence * rng.randn(Np)
            velocity(chi, phi)
            position(self.beam_size * u * np.cos(t), self.beam_size * u * np.sin(t))
        elif bt == 'square':
            assert isinstance(self.beam_size, _VALID_TYPES), \
                "\nReceived beam_size of shape" + str(np.shape(self.beam_size)) + "expected a float."
            t = 2 * rng.rand(Np) - 1.0
            u = 2 * rng.rand(Np) - 1.0
            phi = np.pi * rng.rand(Np)
            chi = self.divergence * rng.randn(Np)
            velocity(chi, phi)
            if d == 'x':
                position(self.beam_size * u, self.beam_size * t)
            elif d == 'z':
                position(self.beam_size * u, self.beam_size * t)
            else:
                position(self.beam_size * u, self.beam_size * t)
        elif bt in ('rectangular', 'rect_trackers'):
            size_dim = len(self.beam_size)
            assert size_dim == 2, ("\nERROR: Must pass a list of length 2 to initialise a rectangular beam,"
                                   + str(size_dim) + "item was passed.")
            t = 2 * rng.rand(Np) - 1.0
            u = 2 * rng.rand(Np) - 1.0
            phi = np.pi * rng.rand(Np)
            chi = self.divergence * rng.randn(Np)
            velocity(chi, phi)
            position(self.beam_size[0] * u, self.beam_size[1] * t)
        elif bt == 'linear':
            assert isinstance(self.beam_size, _VALID_TYPES), \
                "\nReceived beam_size of shape" + str(np.shape(self.beam_size)) + "expected a float."
            t = 2 * rng.rand(Np) - 1.0
            chi = self.divergence * rng.randn(Np)
            s0[3], s0[4], s0[5] = c * np.sin(chi), 0.0, c * np.cos(chi)
            s0[0], s0[1], s0[2] = self.beam_size * t, 0.0, ne_extent
        elif bt == 'even':
            raise NotImplementedError("beam_type 'even' produces no rays in the reference (src/core/beam.py:255-272)")
        else:
            raise ValueError("\nself.beam_type unrecognised! Accepted args: circular, square, rectangular, linear, "
                             "even, rect_trackers.")
        self.s0 = s0.astype(np.float32)

    def save_rays_pos(self, fn=None):
        """Save s0 as .npy (src/core/beam.py:348-370)."""
        from datetime import datetime
        if fn is None:
            fn = '{} rays.npy'.format(datetime.now().strftime("%Y-%m-%d_%H-%M-%S"))
        else:
            fn = '{}.npy'.format(fn)
        with open(fn, 'wb') as f:
            np.save(f, self.s0)
