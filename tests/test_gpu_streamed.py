"""solve / trace_and_save_depths stream the rays through the device in chunks
on two streams. Every chunking must give bitwise the results of one chunk,
for numpy, pinned-host and device ray sources and both precisions."""
import types

import numpy as np
import pytest
import torch

from sloth_b200 import workloads
from sloth_b200.core.propagator import solve, trace_and_save_depths

pytestmark = pytest.mark.gpu

L = 5e-3
N_RAYS = 50_000


def _domain(n=48, inv_brems=True):
    ne = workloads.kolmogorov_box(n, L=L, mean=1e25, rms=0.2, seed=7).numpy().astype(np.float32)
    c1 = np.linspace(-L / 2, L / 2, n).astype(np.float32)
    return types.SimpleNamespace(ne=ne, x=c1, y=c1, z=c1, probing_direction='z',
                                 lengths=np.array([L] * 3, np.float32), dims=np.array([n] * 3), Np_total=None,
                                 inv_brems=inv_brems, Te=np.float32(20.0), Z=np.float32(1.0), region_count=1,
                                 ray_batch_count=1)


def _rays(kind, dtype=torch.float32):
    r = workloads.gaussian_beam(N_RAYS, waist=1.5e-3, L=L, seed=8, dtype=dtype)
    if kind == "numpy":
        return r.numpy()
    if kind == "pinned":
        return r.pin_memory()
    return r.to("cuda")


def _same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape and a.dtype == b.dtype
    assert np.array_equal(np.ascontiguousarray(a).view(np.uint8), np.ascontiguousarray(b).view(np.uint8))


@pytest.mark.parametrize("precision", ["f32", "f64"])
@pytest.mark.parametrize("kind", ["numpy", "pinned", "device"])
def test_solve_chunks_bitwise(precision, kind):
    dom = _domain()
    rays = _rays(kind)
    kw = dict(lwl=532e-9, verbose=False, detector_plane=L / 2, return_extras=True, precision=precision)
    one = solve(rays, dom, L, chunk_rays=N_RAYS, **kw)
    for cs in (7_001, 16_384):          # ragged last chunk, both lanes used repeatedly
        many = solve(rays, dom, L, chunk_rays=cs, **kw)
        for a, b in zip(one[:2], many[:2]):
            _same(a, b)
        for k in ("phase", "status", "steps"):
            _same(one[3][k], many[3][k])
        assert one[3]["total_steps"] == many[3]["total_steps"] > N_RAYS


def test_solve_f64_rays_into_f32_trace():
    """float64 host rays are converted on the device chunk by chunk, as the
    one-shot path converts them."""
    dom = _domain(inv_brems=False)
    r64 = _rays("numpy", torch.float64)
    kw = dict(lwl=532e-9, verbose=False, detector_plane=L / 2, precision="f32")
    a = solve(r64, dom, L, chunk_rays=9_999, **kw)
    b = solve(r64.astype(np.float32), dom, L, chunk_rays=N_RAYS, **kw)
    _same(a[0], b[0])
    assert a[1] is None and b[1] is None


def test_save_depths_and_raw_results_chunks_bitwise():
    dom = _domain()
    rays = _rays("pinned")
    one = trace_and_save_depths(rays, dom, 1e-3, 4e-3, None, lwl=532e-9, verbose=False, return_extras=True,
                                chunk_rays=N_RAYS)
    many = trace_and_save_depths(rays, dom, 1e-3, 4e-3, None, lwl=532e-9, verbose=False, return_extras=True,
                                 chunk_rays=12_345)
    assert len(one["jvec"]) == len(many["jvec"]) == 5
    for k in ("jvec", "amplitude", "phase"):
        for a, b in zip(one[k], many[k]):
            _same(a, b)
    _same(one["status"], many["status"])
    kw = dict(lwl=532e-9, verbose=False, return_raw_results=True, save_points_per_region=4)
    ra = solve(rays, dom, L, chunk_rays=N_RAYS, **kw)[0][0]
    rb = solve(rays, dom, L, chunk_rays=11_111, **kw)[0][0]
    _same(ra.ys, rb.ys)


def test_empty_and_tiny_inputs():
    dom = _domain(n=24)
    kw = dict(lwl=532e-9, verbose=False, detector_plane=L / 2, return_extras=True)
    rf, amp, _, ex = solve(np.zeros((6, 0), np.float32), dom, L, **kw)
    assert rf.shape == (4, 0) and amp.shape == (0,) and ex["total_steps"] == 0
    rays = _rays("numpy")[:, :3]
    a = solve(rays, dom, L, chunk_rays=1, **kw)
    b = solve(rays, dom, L, **kw)
    _same(a[0], b[0])
    _same(a[3]["phase"], b[3]["phase"])
