"""The allocation-free FP32 tracer, sloth_trace_f32_noalloc, called through the C ABI.

It serves callers that cannot allocate device memory (e.g. an XLA FFI
handler inside a JAX program, where XLA owns the device memory), so its
scratch lives in a fixed array inside the library. Two calls in a row, of
different sizes and inputs, must each give bitwise what sloth_trace_f32
(with a caller workspace) gives: both run the same tracer on the same
inputs, and each ray's arithmetic does not depend on the scratch layout.
The file is named to be collected last.
"""
import math

import numpy as np
import pytest
import torch

from sloth_b200 import _capi, runtime, workloads
from sloth_b200.core import physics

pytestmark = pytest.mark.gpu

L = 5e-3


def _params(grid, sched):
    p = _capi.SlothTraceParams()
    p.omega = grid.omega
    p.dtau = sched.dtau
    p.first_save, p.save_every, p.n_saves = sched.first_save, max(1, sched.save_every), sched.n_saves
    p.probing_axis, p.project_to_plane, p.plane = 2, 1, L / 2
    p.inv_brems = 1
    p.kappa_q2, p.coulomb_log_w, p.ope_ratio2 = physics.kappa_factors(20.0, 1.0, grid.omega)
    p.q_max = grid.q_max
    return p


def _outputs(n, S, dev):
    o = {"jones": torch.empty((S, 4, n), device=dev), "phase": torch.empty((S, n), dtype=torch.float64, device=dev),
         "amp": torch.empty((S, n), device=dev), "status": torch.empty(n, dtype=torch.uint8, device=dev),
         "steps": torch.empty(n, dtype=torch.int32, device=dev), "total_steps": torch.empty(1, dtype=torch.int64, device=dev)}
    s = _capi.SlothTraceOutputs()
    for k, t in o.items():
        setattr(s, k, t.data_ptr())
    return o, s


def _trace(entry, grid, rays, sched):
    lib = _capi.load()
    n = rays.shape[1]
    o, s = _outputs(n, sched.n_saves, rays.device)
    p = _params(grid, sched)
    stream = torch.cuda.current_stream().cuda_stream
    if entry == "workspace":
        ws = torch.empty(lib.sloth_trace_workspace_bytes(n), dtype=torch.uint8, device=rays.device)
        rc = lib.sloth_trace_f32(grid.desc, grid.data.data_ptr(), p, rays.data_ptr(), n, s, ws.data_ptr(),
                                 ws.numel(), stream)
    else:
        rc = lib.sloth_trace_f32_noalloc(grid.desc, grid.data.data_ptr(), p, rays.data_ptr(), n, s, stream)
    _capi.check(rc, entry)
    torch.cuda.synchronize()
    return {k: v.cpu() for k, v in o.items()}


def _bits(t):
    """The tensor's bit patterns (NaN compares equal to the same NaN)."""
    return t.view({torch.float32: torch.int32, torch.float64: torch.int64}.get(t.dtype, t.dtype))


def _compare(a, b):
    for k in ("jones", "phase", "amp", "status", "steps", "total_steps"):
        assert torch.equal(_bits(a[k]), _bits(b[k])), k
    assert int(a["total_steps"][0]) == int(b["steps"].long().sum())


def test_noalloc_matches_workspace_entry_point_twice():
    dev = torch.device("cuda", 0)
    n = 48
    h = L / (n - 1)
    omega = physics.omega_of(532e-9)
    ne = workloads.kolmogorov_box(n, L=L, seed=21, device=dev)
    grid = runtime.pack_grid(ne, (-L / 2,) * 3, (h,) * 3, omega, precision="f32")
    first = (workloads.gaussian_beam(30000, waist=2e-3, L=L, seed=22, device=dev),
             runtime.schedule_times([math.sqrt(8.0) * L], (h, h, h)))
    second = (workloads.gaussian_beam(7001, waist=1e-3, L=L, seed=23, jitter=2e-3, device=dev),
              runtime.schedule_times(np.linspace(0.0, L, 4), (h, h, h)))
    for rays, sched in (first, second):
        rays = rays.contiguous()
        got = _trace("noalloc", grid, rays, sched)
        ref = _trace("workspace", grid, rays, sched)
        _compare(got, ref)


def test_noalloc_rejects_too_many_rays():
    lib = _capi.load()
    g = _capi.grid_desc((8, 8, 8), (0, 0, 0), (1e-4,) * 3)
    rc = lib.sloth_trace_f32_noalloc(g, None, _capi.SlothTraceParams(), None, _capi.SLOTH_NOALLOC_MAX_RAYS + 1,
                                     _capi.SlothTraceOutputs(), None)
    assert rc == _capi.SLOTH_ERR_TOO_LARGE


def test_noalloc_at_its_maximum_size():
    """Exactly SLOTH_NOALLOC_MAX_RAYS rays: the keys, permutation and sorted
    keys fill the fixed scratch to its last byte, and the results equal the
    workspace entry point's."""
    n_max = _capi.SLOTH_NOALLOC_MAX_RAYS    # a scratch too small would fail with WORKSPACE_TOO_SMALL
    dev = torch.device("cuda", 0)
    n = 32
    h = L / (n - 1)
    omega = physics.omega_of(532e-9)
    ne = workloads.kolmogorov_box(n, L=L, seed=31, device=dev)
    grid = runtime.pack_grid(ne, (-L / 2,) * 3, (h,) * 3, omega, precision="f32")
    rays = workloads.gaussian_beam(n_max, waist=2e-3, L=L, seed=32, device=dev).contiguous()
    sched = runtime.schedule_times(np.linspace(0.0, L, 2), (h, h, h))
    _compare(_trace("noalloc", grid, rays, sched), _trace("workspace", grid, rays, sched))
