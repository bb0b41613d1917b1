"""Probing beam generated on the GPU (K7, sloth_beam_*): against the numpy
restatement of its generator, invariance to how the rays are split across
calls, the distributions of the reference's Beam, and the Beam(device=...)
mirror."""
import ctypes

import numpy as np
import pytest
import torch

from oracle import beam_np
from sloth_b200 import _capi
from sloth_b200.core.beam import Beam

pytestmark = pytest.mark.gpu

C = 299792458.0


def _kernel(beam_type, axis, size, div, extent, seed, n, first_id=0, precision="f64"):
    p = _capi.SlothBeamParams()
    p.beam_type, p.probing_axis = beam_type, axis
    p.size[0], p.size[1] = size
    p.divergence, p.ne_extent, p.seed, p.first_id = div, extent, seed, first_id
    dt = torch.float64 if precision == "f64" else torch.float32
    out = torch.empty((6, n), dtype=dt, device="cuda")
    fn = _capi.load().sloth_beam_f64 if precision == "f64" else _capi.load().sloth_beam_f32
    _capi.check(fn(ctypes.byref(p), n, _capi.ptr(out), None))
    return out.cpu().numpy()


@pytest.mark.parametrize("beam_type", [0, 1, 2, 3])
@pytest.mark.parametrize("axis", [0, 1, 2])
def test_kernel_matches_restated_generator(beam_type, axis):
    if beam_type == 3 and axis != 2:
        pytest.skip("the linear beam is laid out along z")
    size, n = (1e-3, 2e-3), 20000
    k = _kernel(beam_type, axis, size, 3e-3, -2.5e-3, 1234, n)
    o = beam_np.beam(beam_type, axis, size, 3e-3, -2.5e-3, 1234, n)
    np.testing.assert_allclose(k[:3], o[:3], rtol=1e-14, atol=1e-18)
    np.testing.assert_allclose(k[3:], o[3:], rtol=1e-14, atol=1e-6)
    f32 = _kernel(beam_type, axis, size, 3e-3, -2.5e-3, 1234, n, precision="f32")
    np.testing.assert_array_equal(f32, k.astype(np.float32))


def test_split_across_calls_is_the_same_beam():
    whole = _kernel(0, 2, (1e-3, 0.0), 1e-3, -2e-3, 7, 10000)
    a = _kernel(0, 2, (1e-3, 0.0), 1e-3, -2e-3, 7, 3333)
    b = _kernel(0, 2, (1e-3, 0.0), 1e-3, -2e-3, 7, 10000 - 3333, first_id=3333)
    np.testing.assert_array_equal(np.concatenate([a, b], axis=1), whole)
    other = _kernel(0, 2, (1e-3, 0.0), 1e-3, -2e-3, 8, 10000)
    assert not np.array_equal(other, whole)


def test_distributions_of_the_reference_beam():
    n, R, div = 1_000_000, 1e-3, 2e-3
    s = _kernel(0, 2, (R, 0.0), div, -2.5e-3, 99, n)
    np.testing.assert_allclose(np.linalg.norm(s[3:], axis=0), C, rtol=1e-12)
    assert (s[2] == -2.5e-3).all()
    r = np.hypot(s[0], s[1])
    assert r.max() <= R
    assert abs((r <= R / 2).mean() - 0.25) < 3e-3           # radius R sqrt(U)
    chi = np.arccos(np.clip(s[5] / C, -1, 1))
    assert abs(np.sqrt((chi ** 2).mean()) - div) < 0.01 * div   # |N(0, div)|
    phi = np.mod(np.arctan2(s[4], s[3]), np.pi)    # azimuth pi U; the sign of chi covers the other half
    assert abs(phi.mean() - np.pi / 2) < 0.01 and abs(phi.std() - np.pi / np.sqrt(12)) < 0.01
    q = _kernel(1, 0, (R, 0.0), div, -2.5e-3, 5, n)
    assert (q[0] == -2.5e-3).all() and np.abs(q[1:3]).max() <= R
    for row in (1, 2):
        assert abs(q[row].mean()) < 5e-6 and abs(q[row].std() - R / np.sqrt(3)) < 5e-6


def test_beam_mirror_on_device():
    b = Beam(5000, [1e-3, 2e-3], 1e-3, 2.5e-3, probing_direction='y', beam_type='rect_trackers', seeded=True,
             device="cuda")
    assert isinstance(b.s0, torch.Tensor) and b.s0.is_cuda and b.s0.dtype == torch.float32
    ref = _kernel(2, 1, (1e-3, 2e-3), 1e-3, -2.5e-3, 42, 5000, precision="f32")
    np.testing.assert_array_equal(b.s0.cpu().numpy(), ref)
    with pytest.raises(NotImplementedError):
        Beam(10, 1e-3, 0.0, 1e-3, beam_type="even", device="cuda")
    with pytest.raises(ValueError):
        Beam(10, 1e-3, 0.0, 1e-3, beam_type="donut", device="cuda")
    p = _capi.SlothBeamParams()
    p.beam_type = 9
    assert _capi.load().sloth_beam_f32(ctypes.byref(p), 4, None, None) == _capi.SLOTH_ERR_INVALID_ARGUMENT
