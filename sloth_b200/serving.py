"""Ray-trace request server over the library's continuous-batching core.

``RayServer`` wraps ``sloth_server_*`` (include/sloth_b200.h): grids stay
resident in an HBM arena sized by the admission budget (LRU by grid key),
jobs are admitted in arrival order as memory and slots free up, and each
``step()`` launches one graph-captured iteration of the persistent FP32
tracer over tiles of all admitted jobs. ``replay()`` drives a server with a
timed request stream (seeded Poisson arrivals) and reports p50/p99 latency
and aggregate ray-steps/s.
"""
from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass, field
from typing import Optional

import numpy as np
import torch

from . import _capi as capi
from . import runtime, workloads
from .core import physics


@dataclass
class Job:
    id: int
    n: int
    n_saves: int
    inv_brems: bool
    arrival: float = 0.0
    state: int = capi.SLOTH_JOB_PENDING
    keep: list = field(default_factory=list)      # buffers the server reads until admission
    out: Optional[dict] = None                    # pinned host results once fetched
    done_at: Optional[float] = None
    request: Optional[object] = None              # the stream request it serves (replay)


class RayServer:
    """Continuous-batching ray-trace server on one GPU.

    budget_bytes: HBM admission budget (the arena is allocated up front).
    tiles_per_step: 1024-ray tiles per iteration (default: four per resident
    tracer CTA, 8 per SM; shorter iterations pay their launch and retire
    overhead too often). quantum: tiles per job per round-robin round.
    """

    def __init__(self, budget_bytes: int, *, max_jobs: int = 256, tiles_per_step: Optional[int] = None,
                 quantum: int = 4, device=None):
        self.device = runtime.require_device(device)
        self.lib = capi.load()
        sms, _, _ = capi.device_info()
        cfg = capi.SlothServerConfig()
        cfg.budget_bytes = int(budget_bytes)
        cfg.max_jobs = int(max_jobs)
        cfg.tiles_per_step = int(tiles_per_step or 8 * sms)
        cfg.quantum = int(quantum)
        cfg.reserved = 0
        h = ctypes.c_void_p()
        capi.check(self.lib.sloth_server_create(ctypes.byref(cfg), ctypes.byref(h)), "sloth_server_create")
        self.handle = h
        self.jobs: dict[int, Job] = {}
        self._qmax: dict[int, float] = {}

    # -- lifecycle ----------------------------------------------------------
    def close(self):
        if self.handle:
            self.lib.sloth_server_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- requests -------------------------------------------------------------
    def submit(self, grid_key: int, ne: Optional[torch.Tensor], origin, spacing, shape, rays: torch.Tensor, *,
               lwl: float = 532e-9, depth: Optional[float] = None, detector_plane: Optional[float] = None,
               inv_brems: bool = False, Te=None, Z=None, n_saves: int = 1, probing_axis: int = 2,
               arrival: Optional[float] = None) -> Job:
        """Queue a trace of `rays` ((6, N) float32, CUDA or pinned CPU) through
        the grid `grid_key`. `ne` (m^-3, CUDA) is needed unless the key is
        resident; the server packs it on admission. The rays are traced to
        c*t = sqrt(8)*depth (depth defaults to the grid's extent along the
        probing axis); with `detector_plane` the final rays are projected to it."""
        omega = physics.omega_of(lwl)
        n_rays = int(rays.shape[1])
        desc = capi.grid_desc(shape, origin, spacing)
        if depth is None:
            depth = spacing[probing_axis] * (shape[probing_axis] - 1)
        T = math.sqrt(8.0) * depth
        sched = runtime.schedule_times(np.linspace(0.0, T, n_saves) if n_saves > 1 else [T], spacing)
        p = capi.SlothTraceParams()
        p.omega = omega
        p.dtau = sched.dtau
        p.first_save, p.save_every, p.n_saves = sched.first_save, max(1, sched.save_every), sched.n_saves
        p.probing_axis = probing_axis
        p.project_to_plane = int(detector_plane is not None)
        p.plane = float(detector_plane or 0.0)
        p.inv_brems = int(inv_brems)
        if inv_brems:
            p.kappa_q2, p.coulomb_log_w, p.ope_ratio2 = physics.kappa_factors(Te, Z, omega)
        else:
            p.kappa_q2, p.coulomb_log_w, p.ope_ratio2 = 0.0, 2.0, physics.ope_ratio2(omega)
        if grid_key not in self._qmax:
            if ne is None:
                raise ValueError("ne is required for a grid key seen for the first time")
            lo, hi = torch.aminmax(ne)
            nc = physics.critical_density(omega)
            self._qmax[grid_key] = (max(float(hi) / nc, 0.0) * (1 + 1e-6), min(float(lo) / nc, 0.0) * (1 + 1e-6))
        p.q_max, p.q_min = self._qmax[grid_key]
        if rays.dtype != torch.float32 or not rays.is_contiguous():
            raise ValueError("rays must be a contiguous float32 (6, N) tensor")
        on_host = rays.device.type == "cpu"
        if on_host and not rays.is_pinned():
            raise ValueError("host rays must be in pinned memory")
        ne_ptr = 0
        ne_f64 = 0
        if ne is not None:
            if ne.device.type != "cuda" or not ne.is_contiguous():
                raise ValueError("ne must be a contiguous CUDA tensor")
            ne_ptr = ne.data_ptr()
            ne_f64 = int(ne.dtype == torch.float64)
        jid = ctypes.c_int(0)
        capi.check(self.lib.sloth_server_submit(self.handle, ctypes.c_uint64(grid_key), desc, ne_ptr, ne_f64, p,
                                                rays.data_ptr(), int(on_host), n_rays, ctypes.byref(jid)),
                   "sloth_server_submit")
        job = Job(jid.value, n_rays, sched.n_saves, bool(inv_brems),
                  arrival=time.perf_counter() if arrival is None else arrival, keep=[ne, rays])
        if n_rays == 0:
            # the server finishes a job without rays at once (FETCHED); its
            # results are empty arrays of the usual shapes
            job.out = self._host_outputs(job)
        self.jobs[job.id] = job
        return job

    def step(self):
        run, pend = ctypes.c_int(0), ctypes.c_int(0)
        capi.check(self.lib.sloth_server_step(self.handle, ctypes.byref(run), ctypes.byref(pend)),
                   "sloth_server_step")
        return run.value, pend.value

    def state(self, job: Job) -> int:
        st = ctypes.c_int(0)
        capi.check(self.lib.sloth_server_job_state(self.handle, job.id, ctypes.byref(st)), "sloth_server_job_state")
        job.state = st.value
        if st.value < 0:
            raise capi.SlothError(st.value, f"job {job.id}")
        if st.value != capi.SLOTH_JOB_PENDING:
            job.keep = []
        return st.value

    @staticmethod
    def _host_outputs(job: Job) -> dict:
        """Host buffers for a job's results (pinned when there is anything to copy)."""
        S, N = job.n_saves, job.n
        pin = N > 0
        o = {"jones": torch.empty((S, 4, N), dtype=torch.float32, pin_memory=pin),
             "phase": torch.empty((S, N), dtype=torch.float64, pin_memory=pin),
             "status": torch.empty(N, dtype=torch.uint8, pin_memory=pin),
             "steps": torch.empty(N, dtype=torch.int32, pin_memory=pin),
             "total_steps": torch.zeros(1, dtype=torch.int64, pin_memory=pin)}
        if job.inv_brems:
            o["amp"] = torch.empty((S, N), dtype=torch.float32, pin_memory=pin)
        return o

    def fetch(self, job: Job):
        """Start downloading a DONE job's results into pinned host buffers."""
        o = self._host_outputs(job)
        dst = capi.SlothTraceOutputs()
        for k, t in o.items():
            setattr(dst, k, t.data_ptr())
        capi.check(self.lib.sloth_server_fetch(self.handle, job.id, dst), "sloth_server_fetch")
        job.out = o

    def release(self, job: Job):
        capi.check(self.lib.sloth_server_release(self.handle, job.id), "sloth_server_release")
        self.jobs.pop(job.id, None)

    def cancel(self, job: Job):
        """Cancel a PENDING, RUNNING or DONE job (sloth_server_cancel): it gets
        no further tiles, and its device memory is released once the
        iterations already holding its tiles have finished."""
        capi.check(self.lib.sloth_server_cancel(self.handle, job.id), "sloth_server_cancel")
        job.keep = []
        job.state = capi.SLOTH_JOB_CANCELLED

    def stats(self) -> dict:
        st = capi.SlothServerStats()
        capi.check(self.lib.sloth_server_stats(self.handle, ctypes.byref(st)), "sloth_server_stats")
        return {k: getattr(st, k) for k, _ in st._fields_}

    def sync(self):
        capi.check(self.lib.sloth_server_sync(self.handle), "sloth_server_sync")

    def run_until_done(self, jobs, timeout: float = 600.0):
        """Step until every job is FETCHED; returns their host results."""
        t_end = time.perf_counter() + timeout
        left = {j.id: j for j in jobs}
        while left:
            self.step()
            for j in list(left.values()):
                st = self.state(j)
                if st == capi.SLOTH_JOB_DONE:
                    self.fetch(j)
                elif st == capi.SLOTH_JOB_FETCHED:
                    j.done_at = time.perf_counter()
                    left.pop(j.id)
            if time.perf_counter() > t_end:
                raise TimeoutError(f"{len(left)} jobs unfinished")
        return {j.id: j.out for j in jobs}


# ---------------------------------------------------------------------------
# Timed request streams
# ---------------------------------------------------------------------------
@dataclass
class Request:
    t: float           # arrival time (s from the start of the stream)
    n: int             # grid points per axis
    kind: str          # 'sinusoid' or 'kolmogorov'
    field_seed: int
    rays: int
    ray_seed: int


def request_stream(n_requests=2000, rate=200.0, sizes=(64, 128, 192, 256, 384), ray_median=2e5, ray_sigma=1.0,
                   ray_min=1e4, ray_max=4e6, field_seeds=2, seed=0):
    """Seeded stream: Poisson arrivals at `rate`, grid size uniform over
    `sizes`, field kind by a fair coin (one of `field_seeds` fields per size and
    kind), ray count lognormal(median, sigma) clipped to [ray_min, ray_max]."""
    rng = np.random.RandomState(seed)
    gaps = rng.exponential(1.0 / rate, n_requests)
    t = np.cumsum(gaps) - gaps[0]
    n = rng.choice(np.asarray(sizes), n_requests)
    kind = np.where(rng.rand(n_requests) < 0.5, "sinusoid", "kolmogorov")
    fs = rng.randint(0, field_seeds, n_requests)
    rays = np.clip(np.exp(np.log(ray_median) + ray_sigma * rng.randn(n_requests)), ray_min, ray_max).astype(np.int64)
    rs = rng.randint(0, 2 ** 31 - 1, n_requests)
    return [Request(float(t[i]), int(n[i]), str(kind[i]), int(fs[i]), int(rays[i]), int(rs[i]))
            for i in range(n_requests)]


def field_for(kind, n, seed, L=5e-3, device="cuda"):
    if kind == "sinusoid":
        return workloads.sinusoid_slab(n, L=L, n0=1e24, device=device)
    return workloads.kolmogorov_box(n, L=L, mean=1e25, rms=0.2, seed=seed, device=device)


def grid_key(kind, n, seed):
    return (0 if kind == "sinusoid" else 1) << 40 | int(n) << 20 | int(seed)


def replay(server: RayServer, requests, *, L=5e-3, lwl=532e-9, Te=20.0, Z=1.0, waist=1.5e-3, fields=None,
           realtime=True, max_seconds=600.0):
    """Drive `server` with `requests`; returns latencies (s), ray-steps and
    timing. Kolmogorov requests trace with inverse bremsstrahlung (Te, Z), the
    sinusoid ones without, as in the single-trace configurations."""
    fields = fields if fields is not None else {}
    for r in requests:
        k = grid_key(r.kind, r.n, r.field_seed)
        if k not in fields:
            fields[k] = field_for(r.kind, r.n, r.field_seed, L=L)
    torch.cuda.synchronize()
    h = lambda n: L / (n - 1)
    t0 = time.perf_counter()
    i = 0
    live = []
    lat, steps = [], 0
    records = []           # (arrival s, grid n, rays, latency s) per request, in completion order
    loop_max = 0.0
    first = None
    while i < len(requests) or live:
        loop_start = time.perf_counter()
        now = loop_start - t0
        while i < len(requests) and (not realtime or requests[i].t <= now):
            r = requests[i]
            rays = workloads.gaussian_beam(r.rays, waist=waist, L=L, seed=r.ray_seed, device="cuda")
            k = grid_key(r.kind, r.n, r.field_seed)
            kol = r.kind == "kolmogorov"
            job = server.submit(k, fields[k], (-L / 2,) * 3, (h(r.n),) * 3, (r.n,) * 3, rays, lwl=lwl,
                                detector_plane=L / 2, inv_brems=kol, Te=Te, Z=Z,
                                arrival=t0 + (r.t if realtime else 0.0))
            job.request = r
            live.append(job)
            first = first if first is not None else job.arrival
            i += 1
        server.step()
        still = []
        for j in live:
            st = server.state(j)
            if st == capi.SLOTH_JOB_DONE:
                server.fetch(j)
                still.append(j)
            elif st == capi.SLOTH_JOB_FETCHED:
                j.done_at = time.perf_counter()
                lat.append(j.done_at - j.arrival)
                rq = getattr(j, "request", None)
                records.append((j.arrival - t0, rq.n if rq else 0, rq.rays if rq else 0, j.done_at - j.arrival))
                steps += int(j.out["total_steps"][0])
                server.release(j)
            else:
                still.append(j)
        live = still
        loop_max = max(loop_max, time.perf_counter() - loop_start)
        if time.perf_counter() - t0 > max_seconds:
            raise TimeoutError("request stream did not finish")
    t_end = time.perf_counter()
    lat = np.asarray(lat)
    return {"latency_s": lat, "p50_ms": float(np.percentile(lat, 50) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3), "mean_ms": float(lat.mean() * 1e3),
            "ray_steps": steps, "seconds": t_end - first, "ray_steps_per_s": steps / (t_end - first),
            "requests": len(lat), "stats": server.stats(), "records": records, "host_loop_max_ms": loop_max * 1e3}
