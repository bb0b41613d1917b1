"""ScalarDomain: the electron-density grid the tracers read.

Mirrors core.domain.ScalarDomain of the reference (src/core/domain.py:27-800):
same constructor signature, attributes the propagator reads (ne, x, y, z,
lengths, dims, probing_direction, Np_total, inv_brems, Te, Z, region_count,
ray_batch_count) and the built-in test profiles. The reference's memory-driven
domain/ray batching is not needed on a B200 (a 512^3 float4 grid is 2.1 GB of
180 GB), so region_count and ray_batch_count are always 1; its VTK export is
outside this package.

Coordinates are float32 linspace(-L/2, L/2, n) as in the reference
(:380-382). ne may be a numpy array, a CPU torch tensor (pin it for fast
uploads) or a CUDA tensor; to_device() keeps a device copy for repeated traces.
"""
from __future__ import annotations

import numpy as np

_VALID_TYPES = (int, float, np.integer, np.floating)
_PROFILES = ("test_null", "test_slab", "test_linear_cos", "test_exponential_cos", "import")


class ScalarDomain:
    def __init__(self, lengths, dims, *, ne_type=None, probing_direction='z', auto_batching=True, iteration=1,
                 region_count=1, leeway_factor=None, coord_backup=None, future_dims=None, extra_info=False,
                 memory_reporting=False, memory_limit=None, Np=None, s=None, s1=None, s2=None, Ly=None,
                 ne_0=None, ne=None, inv_brems=False, Te=None, Z=None):
        self.s, self.s1, self.s2, self.Ly, self.ne_0 = s, s1, s2, Ly, ne_0
        self.ne = ne
        if probing_direction not in ('x', 'y', 'z'):
            raise AssertionError("Invalid entry for probing_direction!")
        self.probing_direction = probing_direction
        self.ne_type = ne_type
        # src/core/domain.py:192-207
        assert not inv_brems or (Te is not None and Z is not None), \
            "\nTe and Z must both be provided when inv_brems=True."
        self.inv_brems = inv_brems
        if Te is not None:
            _Te = np.asarray(Te, dtype=np.float32)
            assert float(np.min(_Te)) > 0.0, (
                "\nTe must be a strictly positive electron temperature in eV "
                "(received a zero or negative value).  Do not pass Te in Kelvin or Joules.")
            self.Te = _Te
        else:
            self.Te = None
        self.Z = np.asarray(Z, dtype=np.float32) if Z is not None else None
        self.leeway_factor = leeway_factor if leeway_factor is not None else 1.1
        self.extra_info = extra_info
        self.memory_reporting = memory_reporting
        self.memory_limit = memory_limit
        self.Np_total = np.int64(Np) if Np is not None else None
        self.ray_batch_count = 1
        self.region_count = 1
        self.coord_backup = None
        self.future_dims = None

        if isinstance(lengths, _VALID_TYPES):
            self.x_length = self.y_length = self.z_length = lengths
            self.lengths = np.array([lengths, lengths, lengths])
        else:
            self.lengths = np.array(lengths)
            if self.lengths.shape != (3,):
                raise Exception('lengths must have len = 3: (x,y,z)')
            self.x_length, self.y_length, self.z_length = self.lengths
        if isinstance(dims, _VALID_TYPES):
            self.x_n = self.y_n = self.z_n = int(dims)
            self.dims = np.array([dims, dims, dims])
        else:
            self.dims = np.array(dims)
            if self.dims.shape != (3,):
                raise Exception('n must have len = 3: (x_n, y_n, z_n)')
            self.x_n, self.y_n, self.z_n = (int(v) for v in self.dims)

        self.x = np.float32(np.linspace(-self.x_length / 2, self.x_length / 2, self.x_n))
        self.y = np.float32(np.linspace(-self.y_length / 2, self.y_length / 2, self.y_n))
        self.z = np.float32(np.linspace(-self.z_length / 2, self.z_length / 2, self.z_n))
        self.coordinates = np.stack([self.x, self.y, self.z], axis=1) if \
            (self.x_n == self.y_n == self.z_n) else None
        self.XX = self.YY = self.ZZ = None
        self._device_ne = None

        if self.ne is None:
            if self.ne_type is not None:
                self.generate_electron_density_profile()
            else:
                self.ne = np.zeros((self.x_n, self.y_n, self.z_n), dtype=np.float32)

    # -- profiles (src/core/domain.py:514-682) --------------------------------
    def _mesh(self):
        return np.meshgrid(self.x.astype(np.float64), self.y.astype(np.float64),
                           self.z.astype(np.float64), indexing='ij')

    def generate_electron_density_profile(self):
        if self.ne_type not in _PROFILES:
            raise AssertionError("\nNo valid profile detected! Ensure passed name is correct or call yourself.")
        if self.ne_type == "test_null":
            self.test_null()
        elif self.ne_type == "test_slab":
            self.test_slab()
        elif self.ne_type == "test_linear_cos":
            self.test_linear_cos()
        elif self.ne_type == "test_exponential_cos" or self.ne_type is None:
            self.test_exponential_cos()
        self.cleanup()

    def test_null(self):
        """Empty cube (:566-577)."""
        self.ne = np.zeros((self.x_n, self.y_n, self.z_n), dtype=np.float32)

    def test_slab(self, *, s=1, ne_0=2e23):
        """ne_0 * (1 + s*x/x_length) (:580-602)."""
        s = self.s if self.s is not None else s
        ne_0 = self.ne_0 if self.ne_0 is not None else ne_0
        XX, _, _ = self._mesh()
        self.ne = (ne_0 * (1.0 + s * XX / self.x_length)).astype(np.float32)

    def test_linear_cos(self, *, s1=0.1, s2=0.1, ne_0=2e23, Ly=1):
        """ne_0 * (1 + s1*x/x_length) * (1 + s2*cos(2 pi y/Ly)) (:605-637)."""
        s1 = self.s1 if self.s1 is not None else s1
        s2 = self.s2 if self.s2 is not None else s2
        ne_0 = self.ne_0 if self.ne_0 is not None else ne_0
        Ly = self.Ly if self.Ly is not None else Ly
        XX, YY, _ = self._mesh()
        self.ne = (ne_0 * (1.0 + s1 * XX / self.x_length) * (1 + s2 * np.cos(2 * np.pi * YY / Ly))).astype(np.float32)

    def test_exponential_cos(self, *, ne_0=1e24, Ly=1e-3, s=-2e-3):
        """ne_0 * 10^(x/s) * (1 + cos(2 pi y/Ly)) (:640-682)."""
        ne_0 = self.ne_0 if self.ne_0 is not None else ne_0
        Ly = self.Ly if self.Ly is not None else Ly
        s = self.s if self.s is not None else s
        XX, YY, _ = self._mesh()
        self.ne = (ne_0 * 10 ** (XX / s) * (1 + np.cos(2 * np.pi * YY / Ly))).astype(np.float32)

    def external_ne(self):
        """Keep the imported ne as it is (:685-696)."""
        return None

    def cleanup(self):
        self.XX = self.YY = self.ZZ = None

    # -- device residency ------------------------------------------------------
    def to_device(self, device=None):
        """Keep a CUDA copy of ne for repeated traces; later edits to self.ne
        are not seen until to_device() is called again."""
        import torch
        ne = self.ne
        if isinstance(ne, np.ndarray):
            ne = torch.from_numpy(np.ascontiguousarray(ne))
        dev = torch.device(device) if device is not None else torch.device("cuda")
        self._device_ne = ne.to(dev).contiguous()
        return self

    def export_scalar_field(self, property: str = 'ne', fname: str = None):
        raise NotImplementedError("VTK export (src/core/domain.py:699-781) is not part of the B200 tracer")
