"""The multi-rank path of the bench (sloth_b200/replicas.py) on CPU: two
gloo ranks on 127.0.0.1. The job's time is the max over ranks and its
ray-steps the sum; each rank gets its own seed; and a rank that leaves
before a collective makes its peer's collective fail within the process
group's short timeout instead of hanging."""
import multiprocessing as mp
import os
import socket
import time

import pytest

from sloth_b200 import replicas


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, port, mode, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2", RANK=str(rank),
                      LOCAL_RANK=str(rank))
    try:
        world, r, local = replicas.rank_env()
        dist = replicas.init(world, None, "gloo", timeout_s=5.0)
        replicas.barrier(dist)
        if mode == "leave" and r == 1:
            q.put((r, "left"))
            q.close()
            q.join_thread()    # the message is out before the process goes
            os._exit(0)        # leaves between steps: nothing of its own in flight
        t0 = time.monotonic()
        try:
            ms, steps = replicas.job_totals(dist, 10.0 + 5.0 * r, 100.0 + r, "cpu")
            q.put((r, (ms, steps, replicas.rank_seed(2024, r))))
            replicas.finish(dist)
        except Exception as e:  # the peer is gone
            q.put((r, ("error", type(e).__name__, time.monotonic() - t0)))
    except Exception as e:
        q.put((rank, ("setup", repr(e))))


def _run(mode):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, port, mode, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = {}
    for _ in range(2):
        r, v = q.get(timeout=90)
        out[r] = v
    for p in ps:
        p.join(timeout=30)
        if p.is_alive():
            p.kill()
    return out


def test_single_process_needs_no_group():
    assert replicas.init(1) is None
    assert replicas.job_totals(None, 12.5, 7, "cpu") == (12.5, 7.0)


def test_two_ranks_reduce_time_and_ray_steps():
    out = _run("ok")
    for r in (0, 1):
        ms, steps, seed = out[r]
        assert ms == 15.0 and steps == 201.0
    assert out[0][2] != out[1][2]


def test_rank_that_leaves_fails_its_peer_quickly():
    out = _run("leave")
    assert out[1] == "left"
    kind, _, waited = out[0]
    assert kind == "error"
    assert waited < 60.0
