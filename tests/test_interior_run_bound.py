"""The tracer skips its per-step face test for runs of steps it has proven to
be interior steps. The proof: with every stage acceleration bounded by B
(cells per step^2), after j unit steps from (p, w)

    |w_j - w| <= j B,   |p_j - p - j w| <= B j^2 / 2,

so the position p_j and the prediction p_j + w_j lie within B (j^2/2 + j) of
the segment from p + w to p + (j + 1) w. This checks the envelope against
the tracer's steps driven by adversarial accelerations (every stage at +-B, chosen at
random or to push one way), in FP64 on the CPU."""
import numpy as np
import pytest


def _rkn_step(p, w, accel):
    """The tracer's unit step (phi = 1), Nystrom's fourth-order
    Runge-Kutta-Nystrom method: stages at p, p + w/2 + A1/8, p + w + A2/2;
    p' = p + w + (A1 + 2 A2)/6, w' = w + (A1 + 4 A2 + A3)/6. `accel` gives
    each stage's A."""
    a1 = accel(p)
    a2 = accel(p + w / 2 + a1 / 8)
    a3 = accel(p + w + a2 / 2)
    return p + w + (a1 + 2 * a2) / 6, w + (a1 + 4 * a2 + a3) / 6


@pytest.mark.parametrize("mode", ["random", "push", "alternate"])
@pytest.mark.parametrize("m", [3, 7, 15, 31, 63, 127])
def test_run_envelope_holds(mode, m):
    rng = np.random.default_rng(1 + m)
    B = 0.03
    for trial in range(200):
        p0 = rng.uniform(-50, 50, 3)
        w0 = rng.uniform(-1, 1, 3)
        sign = rng.choice([-1.0, 1.0], 3)
        k = [0]

        def accel(_x):
            k[0] += 1
            if mode == "random":
                return B * rng.choice([-1.0, 1.0], 3)
            if mode == "push":
                return B * sign
            return B * sign * (1.0 if (k[0] // 4) % 2 == 0 else -1.0)

        p, w = p0.copy(), w0.copy()
        for j in range(1, m + 1):
            p, w = _rkn_step(p, w, accel)
            dev = B * (j * j / 2 + j)
            assert np.all(np.abs(w - w0) <= j * B * (1 + 1e-12))
            assert np.all(np.abs(p - p0 - j * w0) <= B * j * j / 2 * (1 + 1e-12) + 1e-12)
            lo = np.minimum(p0 + w0, p0 + (m + 1) * w0) - dev - 1e-12
            hi = np.maximum(p0 + w0, p0 + (m + 1) * w0) + dev + 1e-12
            for x in (p, p + w):
                assert np.all(x >= lo) and np.all(x <= hi), (trial, j)


def test_push_reaches_the_position_bound():
    """The position bound is attained by a constant push, so it cannot be
    tightened."""
    B, m = 0.03, 31
    p, w = np.zeros(3), np.zeros(3)
    for _ in range(m):
        p, w = _rkn_step(p, w, lambda _x: np.full(3, B))
    assert np.allclose(p, B * m * m / 2) and np.allclose(w, B * m)
