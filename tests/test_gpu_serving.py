"""Request server: continuous batching of mixed jobs, HBM-budget admission,
grid residency, and results that are the same alone and in the mix."""
import math

import numpy as np
import pytest
import torch

from sloth_b200 import _capi, runtime, serving, workloads
from sloth_b200.core import physics

pytestmark = pytest.mark.gpu

L = 5e-3
LWL = 532e-9


def _job_specs():
    # (kind, n, rays, seed): mixed grid sizes, ray counts and tracer modes
    return [("kolmogorov", 48, 5000, 1), ("sinusoid", 64, 3000, 2), ("kolmogorov", 32, 20000, 3),
            ("sinusoid", 40, 1500, 4), ("kolmogorov", 48, 700, 5), ("sinusoid", 64, 12000, 6)]


def _fields(specs):
    return {serving.grid_key(k, n, 0): serving.field_for(k, n, 0, L=L) for k, n, _, _ in specs}


def _submit(srv, fields, kind, n, nrays, seed):
    rays = workloads.gaussian_beam(nrays, waist=2e-3, L=L, seed=seed, jitter=1e-3, device="cuda")
    key = serving.grid_key(kind, n, 0)
    h = L / (n - 1)
    kol = kind == "kolmogorov"
    return srv.submit(key, fields[key], (-L / 2,) * 3, (h,) * 3, (n,) * 3, rays, lwl=LWL, detector_plane=L / 2,
                      inv_brems=kol, Te=20.0, Z=1.0), rays


def _direct(fields, kind, n, rays):
    """The same trace through the single-trace entry point."""
    key = serving.grid_key(kind, n, 0)
    h = L / (n - 1)
    g = runtime.pack_grid(fields[key], (-L / 2,) * 3, (h,) * 3, physics.omega_of(LWL))
    sched = runtime.schedule_times([math.sqrt(8.0) * (L)], (h, h, h))
    kol = kind == "kolmogorov"
    out = runtime.trace(g, rays, sched, project=True, plane=L / 2, inv_brems=kol, Te=20.0, Z=1.0)
    torch.cuda.synchronize()
    return {k: v.cpu() for k, v in out.items()}


def _same(a, b):
    assert torch.equal(a["jones"], b["jones"])
    assert torch.equal(a["phase"], b["phase"])
    assert torch.equal(a["steps"], b["steps"]) and torch.equal(a["status"], b["status"])
    if "amp" in b:
        assert torch.equal(a["amp"], b["amp"])
    assert int(a["total_steps"][0]) == int(b["total_steps"][0])


def test_results_same_alone_and_in_the_mix():
    specs = _job_specs()
    fields = _fields(specs)
    with serving.RayServer(2 << 30, tiles_per_step=64, quantum=2) as srv:
        alone = []
        for kind, n, nr, seed in specs:
            job, rays = _submit(srv, fields, kind, n, nr, seed)
            srv.run_until_done([job])
            alone.append((job.out, rays))
            srv.release(job)
        mixed = [_submit(srv, fields, kind, n, nr, seed)[0] for kind, n, nr, seed in specs]
        srv.run_until_done(mixed)
        st = srv.stats()
        assert st["grid_packs"] == len({(k, n) for k, n, _, _ in specs})   # grids stayed resident
    for (kind, n, _, _), (a, rays), m in zip(specs, alone, mixed):
        _same(m.out, a)
        _same(a, _direct(fields, kind, n, rays))


def test_budget_admission_and_eviction():
    # an 80^3 grid (8.2 MB) and a 96^3 grid (14.2 MB) with their jobs (~2.8 MB
    # each) do not fit in 24 MB together: the 96^3 jobs wait until the 80^3
    # jobs are done, and the idle 80^3 grid is evicted to make room
    specs = [("kolmogorov", 80, 40000, s) for s in range(3)] + [("sinusoid", 96, 40000, s) for s in range(3)]
    fields = {}
    for k, n, _, _ in specs:
        fields[serving.grid_key(k, n, 0)] = serving.field_for(k, n, 0, L=L)
    budget = 24 << 20
    with serving.RayServer(budget, tiles_per_step=32) as srv:
        jobs = [_submit(srv, fields, k, n, nr, seed) for k, n, nr, seed in specs]
        res = srv.run_until_done([j for j, _ in jobs])
        st = srv.stats()
        assert st["arena_used"] <= st["budget_bytes"]
        assert st["jobs_done"] == len(specs) and st["jobs_failed"] == 0
        assert st["grid_evictions"] >= 1
    for (kind, n, _, _), (job, rays) in zip(specs, jobs):
        _same(res[job.id], _direct(fields, kind, n, rays))


def test_job_that_can_never_fit_is_refused():
    fields = {serving.grid_key("sinusoid", 128, 0): serving.field_for("sinusoid", 128, 0, L=L)}
    with serving.RayServer(16 << 20) as srv:
        with pytest.raises(_capi.SlothError) as e:
            _submit(srv, fields, "sinusoid", 128, 1000, 0)     # 128^3 grid = 33.5 MB > 16 MB
        assert e.value.code == _capi.SLOTH_ERR_TOO_LARGE


def test_short_request_stream():
    reqs = serving.request_stream(40, rate=400.0, sizes=(32, 48, 64), ray_median=5e3, ray_min=500, ray_max=4e4,
                                  seed=3)
    with serving.RayServer(4 << 30) as srv:
        res = serving.replay(srv, reqs)
    assert res["requests"] == 40
    assert res["p99_ms"] >= res["p50_ms"] > 0
    assert res["ray_steps"] > 0 and res["stats"]["iterations"] >= 1


def test_dense_job_in_the_mix_with_fast_path_jobs():
    """A dense job (near 0.4 nc: its accelerations exceed the interior
    sampling limit) shares the server's kernels with jobs that take the
    interior fast path. Each job's rays must be bitwise its single-trace
    rays, whose dense trace takes interior runs with the grid test."""
    specs = [("kolmogorov", 48, 5000, 1), ("sinusoid", 64, 3000, 2)]
    fields = _fields(specs)
    n = 40
    h = L / (n - 1)
    dkey = serving.grid_key("kolmogorov", n, 99)
    fields[dkey] = workloads.kolmogorov_box(n, L=L, mean=1.5e27, rms=0.2, seed=9, device="cuda")
    rays_d = workloads.gaussian_beam(4000, waist=2e-3, L=L, seed=7, jitter=1e-3, device="cuda")
    with serving.RayServer(2 << 30, tiles_per_step=64, quantum=2) as srv:
        jobs = [_submit(srv, fields, k, nn, nr, s) for k, nn, nr, s in specs]
        jd = srv.submit(dkey, fields[dkey], (-L / 2,) * 3, (h,) * 3, (n,) * 3, rays_d, lwl=LWL,
                        detector_plane=L / 2, inv_brems=True, Te=20.0, Z=1.0)
        srv.run_until_done([j for j, _ in jobs] + [jd])
        outs = [j.out for j, _ in jobs] + [jd.out]
    for (kind, nn, _, _), (job, rays), out in zip(specs, jobs, outs):
        _same(out, _direct(fields, kind, nn, rays))
    g = runtime.pack_grid(fields[dkey], (-L / 2,) * 3, (h,) * 3, physics.omega_of(LWL))
    sched = runtime.schedule_times([math.sqrt(8.0) * L], (h, h, h))
    assert 0.5 * (sched.dtau / h) ** 2 * (g.q_max - min(g.q_min, 0.0)) > 0.03
    direct = runtime.trace(g, rays_d, sched, project=True, plane=L / 2, inv_brems=True, Te=20.0, Z=1.0)
    torch.cuda.synchronize()
    _same(outs[-1], {k: v.cpu() for k, v in direct.items()})


def test_job_without_rays_in_the_mix():
    """A job of zero rays finishes at once with empty results of the usual
    shapes; the job submitted beside it is unaffected."""
    specs = [("kolmogorov", 32, 3000, 7)]
    fields = _fields(specs)
    with serving.RayServer(1 << 30) as srv:
        kind, n, nr, seed = specs[0]
        job, rays = _submit(srv, fields, kind, n, nr, seed)
        h = L / (n - 1)
        key = serving.grid_key(kind, n, 0)
        empty = srv.submit(key, fields[key], (-L / 2,) * 3, (h,) * 3, (n,) * 3,
                           torch.empty((6, 0), dtype=torch.float32, device="cuda"), lwl=LWL,
                           detector_plane=L / 2, inv_brems=True, Te=20.0, Z=1.0, n_saves=3)
        res = srv.run_until_done([job, empty])
        assert srv.state(empty) == _capi.SLOTH_JOB_FETCHED
    e = res[empty.id]
    assert e["jones"].shape == (3, 4, 0) and e["phase"].shape == (3, 0) and e["amp"].shape == (3, 0)
    assert e["status"].shape == (0,) and int(e["total_steps"][0]) == 0
    _same(res[job.id], _direct(fields, kind, n, rays))


def test_arrivals_while_others_run():
    """Jobs B and C arrive after job A's first iteration has been launched and
    while A is still RUNNING; they are admitted into the following
    iterations beside A's remaining tiles. Every result is bitwise the job's
    single-trace result."""
    specs = [("kolmogorov", 48, 40000, 11), ("sinusoid", 64, 6000, 12), ("kolmogorov", 32, 9000, 13)]
    fields = _fields(specs)
    with serving.RayServer(2 << 30, tiles_per_step=8, quantum=1) as srv:
        a, rays_a = _submit(srv, fields, *specs[0])
        srv.step()                                   # admits A, launches its first iteration
        assert srv.state(a) == _capi.SLOTH_JOB_RUNNING
        late = [_submit(srv, fields, *sp) for sp in specs[1:]]
        overlap = False
        left = {a.id: a, **{j.id: j for j, _ in late}}
        while left:
            srv.step()
            states = {j.id: srv.state(j) for j in left.values()}
            if states.get(a.id) == _capi.SLOTH_JOB_RUNNING and any(
                    states.get(j.id) == _capi.SLOTH_JOB_RUNNING for j, _ in late):
                overlap = True
            for jid, st in states.items():
                if st == _capi.SLOTH_JOB_DONE:
                    srv.fetch(left[jid])
                elif st == _capi.SLOTH_JOB_FETCHED:
                    left.pop(jid)
        assert overlap, "no late job ran beside A"
        assert srv.stats()["iterations"] >= 5
    _same(a.out, _direct(fields, specs[0][0], specs[0][1], rays_a))
    for (kind, n, _, _), (j, rays) in zip(specs[1:], late):
        _same(j.out, _direct(fields, kind, n, rays))


def test_cancel_pending_running_and_done_jobs():
    """One table slot: A runs while B waits. A is cancelled mid-run (no
    further tiles; its memory is released after its in-flight iterations
    finish), B is cancelled while PENDING and never runs, C is traced after
    them and matches its single-trace result bitwise, D is cancelled once
    DONE. At the end the arena holds only the resident grids."""
    specs = [("kolmogorov", 48, 60000, 21), ("kolmogorov", 48, 5000, 22), ("kolmogorov", 48, 7000, 23),
             ("kolmogorov", 48, 3000, 24)]
    fields = _fields(specs)
    grid_bytes = 48 ** 3 * 16
    with serving.RayServer(1 << 30, max_jobs=1, tiles_per_step=4, quantum=1) as srv:
        a, _ = _submit(srv, fields, *specs[0])
        b, _ = _submit(srv, fields, *specs[1])
        srv.step()
        assert srv.state(a) == _capi.SLOTH_JOB_RUNNING and srv.state(b) == _capi.SLOTH_JOB_PENDING
        srv.cancel(b)
        srv.step()
        srv.cancel(a)
        assert srv.state(a) == _capi.SLOTH_JOB_CANCELLED and srv.state(b) == _capi.SLOTH_JOB_CANCELLED
        c, rays_c = _submit(srv, fields, *specs[2])
        res = srv.run_until_done([c])
        srv.sync()
        srv.step()                                    # retires A's last iterations
        st = srv.stats()
        assert st["cancelled_pending_free"] == 0 and st["jobs_cancelled"] == 2
        assert st["arena_used"] == grid_bytes
        d, _ = _submit(srv, fields, *specs[3])
        while srv.state(d) != _capi.SLOTH_JOB_DONE:
            srv.step()
        assert srv.stats()["arena_used"] > grid_bytes
        srv.cancel(d)
        assert srv.state(d) == _capi.SLOTH_JOB_CANCELLED
        st = srv.stats()
        assert st["arena_used"] == grid_bytes and st["jobs_cancelled"] == 3
        assert st["jobs_admitted"] == 3                # B never ran
        for j in (a, b, d):
            srv.release(j)
    _same(res[c.id], _direct(fields, specs[2][0], specs[2][1], rays_c))


def test_injected_allocation_failure_at_create():
    """Each of sloth_server_create's allocations, made to fail in turn, ends
    the create with SLOTH_ERR_OUT_OF_MEMORY and releases everything it had
    allocated; a server created afterwards works."""
    lib = _capi.load()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    n_allocs = lib.sloth_server_inject_alloc_failure(0)
    assert n_allocs >= 5
    for k in range(1, n_allocs + 1):
        lib.sloth_server_inject_alloc_failure(k)
        with pytest.raises(_capi.SlothError) as e:
            serving.RayServer(256 << 20, tiles_per_step=16)
        assert e.value.code == _capi.SLOTH_ERR_OUT_OF_MEMORY, k
    lib.sloth_server_inject_alloc_failure(0)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert abs(free0 - free1) < (64 << 20)            # the 256 MB arena was released every time
    specs = [("sinusoid", 40, 2000, 31)]
    fields = _fields(specs)
    with serving.RayServer(256 << 20, tiles_per_step=16) as srv:
        job, rays = _submit(srv, fields, *specs[0])
        res = srv.run_until_done([job])
    _same(res[job.id], _direct(fields, specs[0][0], specs[0][1], rays))
