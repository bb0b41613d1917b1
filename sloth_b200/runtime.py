"""Device runtime over the C ABI: device-resident grids, trace launches,
workspaces and output buffers, all as torch CUDA tensors.

Every compute call goes through ``libsloth_b200.so``; this module only owns
memory and streams. There is no CPU path: on a machine without an sm_100
device the library returns an error and ``SlothError`` is raised.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Optional

import numpy as np
import torch

from . import _capi as capi
from .core import physics

C = physics.C


def _stream_ptr(stream) -> int:
    if stream is None:
        return int(torch.cuda.current_stream().cuda_stream)
    return int(stream.cuda_stream)


def require_device(device=None) -> torch.device:
    """The CUDA device to run on; raises if there is none (no CPU fallback)."""
    if not torch.cuda.is_available():
        raise capi.SlothError(capi.SLOTH_ERR_NO_DEVICE, "sloth_b200 needs a CUDA device (B200, sm_100)")
    capi.load()
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    return dev


def uniform_axis(coords) -> tuple[float, float, int]:
    """(origin, spacing, n) of a uniformly spaced coordinate array; raises
    NotImplementedError for a non-uniform one (the tracers index a uniform grid)."""
    c = np.asarray(coords, dtype=np.float64).ravel()
    n = c.size
    if n < 2:
        raise ValueError("each grid axis needs at least 2 points")
    h = (c[-1] - c[0]) / (n - 1)
    if not h > 0:
        raise ValueError("grid coordinates must be increasing")
    dev = np.max(np.abs(c - (c[0] + h * np.arange(n))))
    if dev > 1e-3 * h:
        raise NotImplementedError("non-uniform grid coordinates are not supported by the B200 tracers")
    return float(c[0]), float(h), n


@dataclass
class DeviceGrid:
    """A packed (c0, dq/du, dq/dv, dq/dw) grid resident in HBM: c0 = n - 1 in
    the trace layout (what the tracers read), c0 = q in the value layout (the
    K0 sampler's)."""
    data: torch.Tensor
    desc: capi.SlothGridDesc
    precision: str
    omega: float
    n: tuple
    origin: tuple
    spacing: tuple
    q_max: float = 0.0         # max of the q channel (ne/nc) over the grid; 0 = unknown
    q_min: float = float("inf")  # a lower bound of min(q, 0) over the grid; inf = unknown
    ne_max: float = float("nan")  # largest ne (m^-3) packed, from the device reduction
    layout: str = "trace"

    @property
    def nc(self) -> float:
        return physics.critical_density(self.omega)

    @property
    def extent_lo(self):
        return tuple(self.origin)

    @property
    def extent_hi(self):
        return tuple(o + h * (k - 1) for o, h, k in zip(self.origin, self.spacing, self.n))


def pack_grid(ne, origin, spacing, omega, *, precision="f32", device=None, stream=None,
              out: Optional[torch.Tensor] = None, ne_scale: Optional[float] = None,
              layout: str = "trace") -> DeviceGrid:
    """K1: pack ne (m^-3, (nx, ny, nz) array or tensor) into a device grid.

    ``ne`` may be a numpy array, a CPU tensor (pinned for a fast copy) or a
    CUDA tensor; float32 and float64 are read as they are. q = ne * ne_scale
    with ne_scale = 1/nc(omega) unless given. ``layout`` 'trace' (the
    tracers' grid) stores n - 1 of the plasma refractive index in channel 0,
    'values' stores q there (for the K0 sampler).
    """
    if layout not in ("trace", "values"):
        raise ValueError("layout must be 'trace' or 'values'")
    dev = require_device(device)
    if isinstance(ne, np.ndarray):
        ne = torch.from_numpy(np.ascontiguousarray(ne))
    if ne.dtype not in (torch.float32, torch.float64):
        ne = ne.to(torch.float32)
    if ne.dim() != 3:
        raise ValueError("ne must be a 3-D (nx, ny, nz) array")
    if ne.device.type != "cuda":
        ne = ne.to(dev, non_blocking=True)
    ne = ne.contiguous()
    n = tuple(int(k) for k in ne.shape)
    desc = capi.grid_desc(n, origin, spacing)
    rb = 4 if precision == "f32" else 8
    nbytes = capi.load().sloth_grid_bytes(desc, rb)
    if nbytes == 0:
        raise ValueError(f"invalid grid {n}")
    if out is None:
        out = torch.empty(nbytes // rb, dtype=torch.float32 if rb == 4 else torch.float64, device=dev)
    scale = 1.0 / physics.critical_density(omega) if ne_scale is None else float(ne_scale)
    lib = capi.load()
    if layout == "trace":
        fn = lib.sloth_grid_pack_trace_f32 if precision == "f32" else lib.sloth_grid_pack_trace_f64
        capi.check(fn(desc, capi.ptr(ne), int(ne.dtype == torch.float64), scale, physics.ope_ratio2(omega),
                      capi.ptr(out), _stream_ptr(stream)), "sloth_grid_pack_trace")
    else:
        fn = lib.sloth_grid_pack_f32 if precision == "f32" else lib.sloth_grid_pack_f64
        capi.check(fn(desc, capi.ptr(ne), int(ne.dtype == torch.float64), scale, capi.ptr(out),
                      _stream_ptr(stream)), "sloth_grid_pack")
    if ne.numel():
        lo, hi = torch.aminmax(ne)
        ne_max = float(hi)
        q_max, q_min = ne_max * scale, float(lo) * scale
    else:
        ne_max, q_max, q_min = 0.0, 0.0, 0.0
    return DeviceGrid(out, desc, precision, float(omega), n, tuple(map(float, origin)), tuple(map(float, spacing)),
                      q_max=max(q_max, 0.0) * (1.0 + 1e-6), q_min=min(q_min, 0.0) * (1.0 + 1e-6), ne_max=ne_max,
                      layout=layout)


def sample(grid: DeviceGrid, points, *, stream=None) -> torch.Tensor:
    """K0: (4, N) interpolated (c0, dq/du, dq/dv, dq/dw) at points (3, N) in
    metres (c0 = q in the value layout)."""
    pts = torch.as_tensor(points, dtype=torch.float64)
    pts = pts.to(grid.data.device).contiguous()
    n = pts.shape[1]
    out = torch.empty((4, n), dtype=grid.data.dtype, device=grid.data.device)
    fn = capi.load().sloth_sample_f32 if grid.precision == "f32" else capi.load().sloth_sample_f64
    capi.check(fn(grid.desc, capi.ptr(grid.data), capi.ptr(pts), n, capi.ptr(out), _stream_ptr(stream)),
               "sloth_sample")
    return out


@dataclass
class Schedule:
    """Fixed-step schedule: every step is dtau (metres of c*t); save j is
    taken after step first_save + j*save_every."""
    dtau: float
    first_save: int
    save_every: int
    n_saves: int

    @property
    def last_step(self) -> int:
        return self.first_save + (self.n_saves - 1) * (self.save_every if self.n_saves > 1 else 0)


def nominal_step(spacing) -> float:
    """Path-length step: half the smallest grid spacing."""
    return 0.5 * min(spacing)


def schedule_times(tau_saves, spacing) -> Schedule:
    """Schedule whose saves land exactly on uniformly spaced c*t values
    tau_saves[j] = tau_saves[0] + j*d (tau_saves[0] is 0 or the only save);
    the step is the largest dtau <= nominal_step that divides d."""
    tau_saves = np.asarray(tau_saves, dtype=np.float64)
    h = nominal_step(spacing)
    if tau_saves.size == 1:
        T = float(tau_saves[0])
        if T <= 0:
            return Schedule(h, 0, 1, 1)
        m = max(1, math.ceil(T / h - 1e-9))
        return Schedule(T / m, m, 1, 1)
    if abs(tau_saves[0]) > 0:
        raise ValueError("multi-save schedules start at t = 0")
    d = float(tau_saves[1] - tau_saves[0])
    m = max(1, math.ceil(d / h - 1e-9))
    return Schedule(d / m, 0, m, int(tau_saves.size))


_ws_cache: dict = {}


def _workspace(n: int, device) -> torch.Tensor:
    need = int(capi.load().sloth_trace_workspace_bytes(n))
    key = (str(device),)
    t = _ws_cache.get(key)
    if t is None or t.numel() < need:
        t = torch.empty(need, dtype=torch.uint8, device=device)
        _ws_cache[key] = t
    return t


def integrator_code(integrator: str) -> int:
    """SLOTH_INTEGRATOR_* of 'rkn' or 'rk4'."""
    codes = {"rkn": capi.SLOTH_INTEGRATOR_RKN, "rk4": capi.SLOTH_INTEGRATOR_RK4}
    if integrator not in codes:
        raise ValueError(f"integrator must be 'rkn' or 'rk4', not {integrator!r}")
    return codes[integrator]


def trace(grid: DeviceGrid, rays: torch.Tensor, sched: Schedule, *, axis=2, project=False, plane=0.0,
          inv_brems=False, Te=None, Z=None, want_state=False, want_phase=True, want_amp=None,
          want_status=True, want_steps=True, stream=None, workspace: Optional[torch.Tensor] = None,
          outputs: Optional[dict] = None, events=None, integrator: str = "rkn") -> dict:
    """K2/K3: trace rays (6, N) (device tensor of the grid's precision).

    ``integrator`` is 'rkn' (fourth-order Runge-Kutta-Nystrom, three field
    samples per step, the default) or 'rk4' (classical RK4, four samples).

    Returns a dict of device tensors: jones [S,4,N], optional state [S,6,N],
    phase [S,N] (float64), amp [S,N], status [N] (uint8), steps [N] (int32),
    total_steps [1] (int64 view of the kernel's counter). ``events`` is an
    optional pair of recorded torch.cuda.Event(enable_timing=True) that the
    library re-records around the tracer kernel alone.
    """
    if grid.layout != "trace":
        raise ValueError("the tracers read grids packed with layout='trace'")
    dtype = torch.float32 if grid.precision == "f32" else torch.float64
    if rays.dtype != dtype or rays.device != grid.data.device or not rays.is_contiguous():
        rays = rays.to(device=grid.data.device, dtype=dtype).contiguous()
    if rays.dim() != 2 or rays.shape[0] != 6:
        raise ValueError("rays must have shape (6, N)")
    n = int(rays.shape[1])
    S = sched.n_saves
    dev = grid.data.device
    if want_amp is None:
        want_amp = inv_brems
    o = outputs if outputs is not None else {}

    def buf(key, shape, dt, want=True):
        if not want:
            o.pop(key, None)
            return None
        t = o.get(key)
        if t is None or tuple(t.shape) != tuple(shape) or t.dtype != dt:
            t = torch.empty(shape, dtype=dt, device=dev)
            o[key] = t
        return t

    jones = buf("jones", (S, 4, n), dtype)
    state = buf("state", (S, 6, n), dtype, want_state)
    phase = buf("phase", (S, n), torch.float64, want_phase)
    amp = buf("amp", (S, n), dtype, want_amp)
    status = buf("status", (n,), torch.uint8, want_status)
    steps = buf("steps", (n,), torch.int32, want_steps)
    total = buf("total_steps", (1,), torch.int64)
    p = capi.SlothTraceParams()
    p.omega = grid.omega
    p.dtau = sched.dtau
    p.first_save = sched.first_save
    p.save_every = max(1, sched.save_every)
    p.n_saves = S
    p.probing_axis = int(axis)
    p.project_to_plane = int(bool(project))
    p.plane = float(plane)
    p.inv_brems = int(bool(inv_brems))
    if inv_brems:
        kq2, clw, ope2 = physics.kappa_factors(Te, Z, grid.omega)
        p.kappa_q2, p.coulomb_log_w, p.ope_ratio2 = kq2, clw, ope2
    else:
        p.kappa_q2, p.coulomb_log_w, p.ope_ratio2 = 0.0, 2.0, physics.ope_ratio2(grid.omega)
    p.q_max = float(grid.q_max)
    p.q_min = float(grid.q_min)
    p.integrator = integrator_code(integrator)
    out = capi.SlothTraceOutputs()
    out.jones = capi.ptr(jones)
    out.state = capi.ptr(state)
    out.phase = capi.ptr(phase)
    out.amp = capi.ptr(amp)
    out.status = capi.ptr(status)
    out.steps = capi.ptr(steps)
    out.total_steps = capi.ptr(total)
    if events is not None:
        out.trace_event_begin = int(events[0].cuda_event)
        out.trace_event_end = int(events[1].cuda_event)
    ws = workspace if workspace is not None else _workspace(n, dev)
    fn = capi.load().sloth_trace_f32 if grid.precision == "f32" else capi.load().sloth_trace_f64
    capi.check(fn(grid.desc, capi.ptr(grid.data), p, capi.ptr(rays), n, out, capi.ptr(ws), ws.numel(),
                  _stream_ptr(stream)), "sloth_trace")
    return o


_lane_cache: dict = {}


def _lanes(dev):
    """Two side streams of the device (created once) for trace_to_host."""
    key = str(dev)
    lanes = _lane_cache.get(key)
    if lanes is None:
        lanes = (torch.cuda.Stream(dev), torch.cuda.Stream(dev))
        _lane_cache[key] = lanes
    return lanes


def _lane_workspace(n: int, dev, lane: int) -> torch.Tensor:
    need = int(capi.load().sloth_trace_workspace_bytes(n))
    key = (str(dev), "lane", lane)
    t = _ws_cache.get(key)
    if t is None or t.numel() < need:
        t = torch.empty(need, dtype=torch.uint8, device=dev)
        _ws_cache[key] = t
    return t


STREAM_CHUNK_RAYS = 1 << 24
STREAM_END_RAYS = 1 << 19


def _chunk_bounds(n: int, cs: int) -> list:
    """Chunk boundaries of n rays for trace_to_host: at most `cs` rays per
    chunk. Above 8 * STREAM_END_RAYS rays (8 * cs when cs is smaller) the
    first and the last chunk hold only that many, because the first chunk's
    copy in and the last chunk's copy out are the only copies no trace hides;
    below it every chunk is alike. Chunks between the ends differ in size by
    one ray at most.

    Each chunk is one trace launch, and a launch costs more than its rays'
    share (its ramp and the tail of its tile queue: at 512^3 with a 3 mm
    waist beam, 3M rays trace at 114 ms per 1e7 rays against 102 ms in one
    launch of 1e7). So the default takes chunks as large as the end chunks'
    traces can hide the middle chunks' copies behind: 1e7 rays go through as
    0.5M, 9M and 0.5M (118 ms for solve() with that beam against 126 ms as
    0.5M, three of 3M and 0.5M)."""
    if n <= 0:
        return [0, 0]

    def split(lo, hi):
        m = hi - lo
        k = max(1, -(-m // cs))
        q, r = divmod(m, k)
        return [lo + i * q + min(i, r) for i in range(k + 1)]

    end = min(cs, STREAM_END_RAYS)
    if n <= 8 * end:
        return split(0, n)
    return [0] + split(end, n - end) + [n]


def trace_to_host(grid: DeviceGrid, rays, sched: Schedule, *, want: dict, chunk_rays: Optional[int] = None,
                  stream=None, **kw):
    """Trace rays (6, N) and return the requested outputs as numpy arrays,
    streaming the rays through the device in chunks.

    ``rays`` is a host or device tensor or a numpy array. ``want`` maps output
    names ("jones", "state", "phase", "amp", "status", "steps") to "all"
    (every save) or "last" (the last save; per-ray outputs ignore it). The
    other keywords are those of ``trace``.

    Chunk c runs on side stream c % 2: its rays are copied in, traced, and
    its outputs copied into pinned host arrays at the chunk's columns. While
    one chunk traces, the other stream's copies run, so the host<->device
    traffic hides under the tracer except for the first chunk's rays and the
    last chunk's outputs. Each ray's arithmetic does not depend on the other
    rays of its launch, so the results are bitwise those of one trace of all
    N rays.

    Returns (dict of numpy arrays, total ray-steps, seconds from the first
    copy to the last output on the host).
    """
    import time

    dtype = torch.float32 if grid.precision == "f32" else torch.float64
    dev = grid.data.device
    src = torch.from_numpy(np.ascontiguousarray(rays)) if not isinstance(rays, torch.Tensor) else rays
    if src.dim() != 2 or src.shape[0] != 6:
        raise ValueError("rays must have shape (6, N)")
    if src.stride(1) != 1:
        src = src.contiguous()
    n = int(src.shape[1])
    S = sched.n_saves
    bounds = _chunk_bounds(n, int(chunk_rays or STREAM_CHUNK_RAYS))
    n_chunks = len(bounds) - 1
    inv_brems = bool(kw.get("inv_brems", False))
    want = {k: v for k, v in want.items() if k != "amp" or inv_brems}

    def host_shape(k):
        rows = {"jones": (4,), "state": (6,)}.get(k, ())
        if k in ("status", "steps"):
            return (n,)
        return ((S,) if want[k] == "all" else ()) + rows + (n,)

    hdt = {"jones": dtype, "state": dtype, "amp": dtype, "phase": torch.float64, "status": torch.uint8,
           "steps": torch.int32}
    host = {k: torch.empty(host_shape(k), dtype=hdt[k], pin_memory=True) for k in want}
    totals = torch.empty(n_chunks, dtype=torch.int64, pin_memory=True)
    cur = stream if stream is not None else torch.cuda.current_stream(dev)
    ready = torch.cuda.Event()
    ready.record(cur)
    lanes = _lanes(dev)
    for lane in lanes:
        lane.wait_event(ready)
    outs = ({}, {})
    stage = [None, None]
    t0 = time.perf_counter()
    for c in range(n_chunks):
        a, b = bounds[c], bounds[c + 1]
        li = c % 2
        lane = lanes[li]
        with torch.cuda.stream(lane):
            m = b - a
            st = stage[li]
            if st is None or st.shape[1] != m or st.dtype != src.dtype:
                st = torch.empty((6, m), dtype=src.dtype, device=dev)
                stage[li] = st
            for r in range(6):
                st[r].copy_(src[r, a:b], non_blocking=True)
            rc = st if src.dtype == dtype else st.to(dtype)
            o = trace(grid, rc, sched, stream=lane, workspace=_lane_workspace(m, dev, li), outputs=outs[li],
                      want_state="state" in want, want_phase="phase" in want, want_amp="amp" in want,
                      want_status="status" in want, want_steps="steps" in want, **kw)
            for k, h in host.items():
                d = o[k]
                if k in ("status", "steps"):
                    h[a:b].copy_(d, non_blocking=True)
                    continue
                if want[k] == "last":
                    d = d[-1]
                    if d.dim() == 1:
                        h[a:b].copy_(d, non_blocking=True)
                    else:
                        for r in range(d.shape[0]):
                            h[r, a:b].copy_(d[r], non_blocking=True)
                    continue
                for s_ in range(S):
                    if d.dim() == 2:
                        h[s_, a:b].copy_(d[s_], non_blocking=True)
                    else:
                        for r in range(d.shape[1]):
                            h[s_, r, a:b].copy_(d[s_, r], non_blocking=True)
            totals[c:c + 1].copy_(o["total_steps"], non_blocking=True)
    for lane in lanes:
        lane.synchronize()
        cur.wait_stream(lane)
    dt = time.perf_counter() - t0
    return {k: h.numpy() for k, h in host.items()}, int(totals.sum()), dt
