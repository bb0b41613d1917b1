"""One solve() job split over two gloo ranks on 127.0.0.1.

Every rank passes the same beam and domain; each traces a contiguous slice
of the rays (slices differ by one ray at most) and every rank returns the
results of all rays in their original order, the total ray-steps summed and
the time the longest over the ranks.

The CUDA kernels cannot run here, so the test replaces the per-rank trace
(runtime.trace_to_host) and the grid pack by a stand-in whose outputs are a
fixed function of each ray. What is tested is the host logic around them:
the slices, the all-gather into ray order and the two reductions. On GPUs the
same code runs the real trace, with the gather over NCCL."""
import multiprocessing as mp
import os
import socket
import types

import numpy as np
import pytest

N_RAYS, N_SAVES = 1001, 3


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rays():
    rng = np.random.default_rng(5)
    r = rng.normal(size=(6, N_RAYS)).astype(np.float32)
    r[5] = 3e8
    return r


def _fake_trace(grid, rays, sched, *, want, chunk_rays=None, stream=None, **kw):
    """Outputs that depend on each ray alone (like the tracer's)."""
    r = np.asarray(rays, dtype=np.float64)
    n = r.shape[1]
    S = sched.n_saves
    out = {}
    for k, mode in want.items():
        if k == "jones":
            j = np.stack([r[0] * 2, r[3], r[1] - 1, r[4]]).astype(np.float32)
            out[k] = np.stack([j + s for s in range(S)]) if mode == "all" else j
        elif k == "amp":
            a = np.exp(-np.abs(r[0])).astype(np.float32)
            out[k] = np.stack([a] * S) if mode == "all" else a
        elif k == "phase":
            out[k] = np.stack([r[1] * (s + 1) for s in range(S)])
        elif k == "status":
            out[k] = (r[2] > 0).astype(np.uint8)
        elif k == "steps":
            out[k] = (np.abs(r[0]) * 100).astype(np.int32)
    total = int((np.abs(r[0]) * 100).astype(np.int32).sum())
    return out, total, 0.5 + 0.25 * n / N_RAYS


def _install_fakes(propagator, runtime):
    runtime.trace_to_host = _fake_trace
    runtime.require_device = lambda device=None: "cpu"
    propagator.device_grid = lambda dom, omega, **k: types.SimpleNamespace(spacing=(1e-4,) * 3)
    runtime.schedule_times = lambda taus, spacing: types.SimpleNamespace(n_saves=len(taus), dtau=1e-5,
                                                                         first_save=0, save_every=1)


def _domain(n=8):
    c = np.linspace(-2.5e-3, 2.5e-3, n).astype(np.float32)
    return types.SimpleNamespace(ne=np.zeros((n, n, n), np.float32), x=c, y=c, z=c, probing_direction='z',
                                 lengths=np.array([5e-3] * 3, np.float32), dims=np.array([n] * 3), Np_total=None,
                                 inv_brems=True, Te=np.float32(20.0), Z=np.float32(1.0))


def _run(group=None):
    from sloth_b200 import runtime
    from sloth_b200.core import propagator
    _install_fakes(propagator, runtime)
    rays = _rays()
    rf, amp, dur, ex = propagator.solve(rays, _domain(), 5e-3, verbose=False, return_extras=True, group=group)
    rf3, _, _, ex3 = propagator.solve(rays, _domain(), 5e-3, verbose=False, return_extras=True,
                                      save_points_per_region=N_SAVES, group=group)
    tsd = propagator.trace_and_save_depths(rays, _domain(), 2e-3, 4e-3, None, verbose=False, group=group)
    return dict(rf=rf, amp=amp, dur=float(dur), phase=ex["phase"], status=ex["status"], steps=ex["steps"],
                total=ex["total_steps"], rf3=rf3, phase3=ex3["phase"], jvec=np.stack(tsd["jvec"]),
                ampl=np.stack(tsd["amplitude"]))


def _rank_main(rank, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2", RANK=str(rank))
    try:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("gloo", rank=rank, world_size=2, timeout=datetime.timedelta(seconds=20))
        out = _run(dist.group.WORLD)
        q.put((rank, out))
        dist.destroy_process_group()
    except Exception as e:
        import traceback
        q.put((rank, ("error", repr(e) + traceback.format_exc())))


def _single_main(q):
    try:
        q.put((-1, _run(None)))
    except Exception as e:
        q.put((-1, ("error", repr(e))))


def test_shard_bounds_cover_the_rays_in_order():
    from sloth_b200 import shard
    for n in (0, 1, 5, 1000, 1001, 2 ** 20 + 3):
        for world in (1, 2, 3, 8):
            b = [shard.shard_bounds(n, world, r) for r in range(world)]
            assert b[0][0] == 0 and b[-1][1] == n
            assert all(b[i][1] == b[i + 1][0] for i in range(world - 1))
            sizes = [hi - lo for lo, hi in b]
            assert max(sizes) - min(sizes) <= 1


def test_solve_split_over_two_ranks_equals_one_process():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    # the stand-ins are installed in child processes only
    ps = [ctx.Process(target=_rank_main, args=(r, port, q)) for r in range(2)]
    ps.append(ctx.Process(target=_single_main, args=(q,)))
    for p in ps:
        p.start()
    out = {}
    for _ in range(3):
        r, v = q.get(timeout=120)
        out[r] = v
    for p in ps:
        p.join(timeout=30)
    assert all(isinstance(v, dict) for v in out.values()), out
    one = out[-1]
    for r in (0, 1):
        got = out[r]
        for k in ("rf", "amp", "phase", "status", "steps", "rf3", "phase3", "jvec", "ampl"):
            assert got[k].shape == one[k].shape, k
            assert np.array_equal(got[k], one[k]), k
        assert got["total"] == one["total"]
        # the longest rank's time: the first rank holds the extra ray
        assert got["dur"] == pytest.approx(0.5 + 0.25 * 501 / N_RAYS)
