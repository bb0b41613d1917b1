"""The detector image's multi-rank path on CPU: two gloo ranks on 127.0.0.1,
each with its own shard of rays. The image must be the sum over ranks, and
ne.grad the gradient of the loss on that summed image with respect to all
rays, on every rank.

The CUDA kernels cannot run here, so the test replaces this process's
forward and backward (sloth_b200.adjoint._image_forward / _image_backward)
by a linear stand-in, image_r = A_r ne with a rank-seeded matrix A_r. What is
tested is the host logic around them: the all-reduce of the image in the
forward, the loss gradient that reaches the backward, and the all-reduce of
the gradient."""
import multiprocessing as mp
import os
import socket

import numpy as np
import torch

N_VOX, N_PX = (3, 4, 5), (6, 7)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _matrix(rank):
    g = torch.Generator().manual_seed(100 + rank)
    return torch.randn(int(np.prod(N_PX)), int(np.prod(N_VOX)), generator=g, dtype=torch.float64)


def _rank_main(rank, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2", RANK=str(rank))
    try:
        import datetime

        import torch.distributed as dist

        from sloth_b200 import adjoint

        dist.init_process_group("gloo", rank=rank, world_size=2, timeout=datetime.timedelta(seconds=20))
        A = _matrix(rank)

        def fake_forward(ne, rays, origin, spacing, omega, spec, precision, stats):
            return (A @ ne.detach().reshape(-1)).reshape(N_PX), {"A": A, "shape": tuple(ne.shape)}

        def fake_backward(state, grad_image):
            return (state["A"].T @ grad_image.reshape(-1)).reshape(state["shape"])

        adjoint._image_forward, adjoint._image_backward = fake_forward, fake_backward
        spec = adjoint.DetectorSpec(window=(0.0, 1.0, 0.0, 1.0), plane=1.0, dtau=0.1, n_px=N_PX)
        ne = torch.linspace(0.5, 2.0, int(np.prod(N_VOX)), dtype=torch.float64).reshape(N_VOX)
        target = torch.full(N_PX, 0.25, dtype=torch.float64)
        x = ne.clone().requires_grad_(True)
        img = adjoint.detector_image(x, torch.zeros(6, 1), spec, origin=(0, 0, 0), spacing=(1, 1, 1), omega=1.0,
                                     group=dist.group.WORLD)
        loss = ((img - target) ** 2).sum()
        loss.backward()
        q.put((rank, (img.detach().numpy(), float(loss), x.grad.numpy())))
        dist.destroy_process_group()
    except Exception as e:
        q.put((rank, ("error", repr(e))))


def test_image_and_gradient_are_summed_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = {}
    for _ in range(2):
        r, v = q.get(timeout=120)
        out[r] = v
    for p in ps:
        p.join(timeout=30)
    assert all(not isinstance(v[0], str) for v in out.values()), out
    # the same computation in one process over both shards
    A = _matrix(0) + _matrix(1)
    ne = np.linspace(0.5, 2.0, int(np.prod(N_VOX)))
    img = A.numpy() @ ne
    resid = img - 0.25
    grad = 2.0 * (A.numpy().T @ resid)
    for r in (0, 1):
        im, loss, g = out[r]
        assert np.allclose(im.reshape(-1), img, rtol=1e-12, atol=1e-12)
        assert np.isclose(loss, float((resid ** 2).sum()), rtol=1e-12)
        assert np.allclose(g.reshape(-1), grad, rtol=1e-12, atol=1e-10)
