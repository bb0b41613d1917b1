"""Test infrastructure only: a numpy restatement of the device beam generator
(sloth_b200/csrc/beam.cu): the same SplitMix64 draws per (seed, ray id,
draw), the same Box-Muller normal, the same placement of the reference's
Beam (src/core/beam.py:57-346) per beam type and probing direction, in
FP64. The uniform draws are bit-identical to the kernel's; the
trigonometry may differ in the last bit."""
from __future__ import annotations

import numpy as np

C = 299792458.0
M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def _splitmix64(z):
    z = z.astype(np.uint64)
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xbf58476d1ce4e5b9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94d049bb133111eb)
    return z ^ (z >> np.uint64(31))


def uniform(seed, ids, k):
    ids = np.asarray(ids, dtype=np.uint64)
    with np.errstate(over="ignore"):
        inner = _splitmix64(ids * np.uint64(8) + np.uint64(k + 1))
        h = _splitmix64(np.uint64(seed) * np.uint64(0x9e3779b97f4a7c15) + inner)
    return (h >> np.uint64(11)).astype(np.float64) * 2.0 ** -53


def beam(beam_type, axis, size, divergence, extent, seed, n, first_id=0):
    ids = np.arange(first_id, first_id + n, dtype=np.uint64)
    u = [uniform(seed, ids, k) for k in range(5)]
    gauss = np.sqrt(-2.0 * np.log(1.0 - u[3])) * np.cos(2.0 * np.pi * u[4])
    chi = divergence * gauss
    phi = np.pi * u[2]
    if beam_type == 0:
        t, r = 2.0 * np.pi * u[0], size[0] * np.sqrt(u[1])
        pa, pb = r * np.cos(t), r * np.sin(t)
    elif beam_type == 3:
        pa, pb = size[0] * (2.0 * u[0] - 1.0), np.zeros(n)
    else:
        pa, pb = size[0] * (2.0 * u[1] - 1.0), (size[0] if beam_type == 1 else size[1]) * (2.0 * u[0] - 1.0)
    s0 = np.zeros((6, n))
    if beam_type == 3:
        s0[0], s0[2] = pa, extent
        s0[3], s0[5] = C * np.sin(chi), C * np.cos(chi)
        return s0
    ca, s1, s2 = C * np.cos(chi), C * np.sin(chi) * np.cos(phi), C * np.sin(chi) * np.sin(phi)
    if axis == 0:
        s0[0], s0[1], s0[2], s0[3], s0[4], s0[5] = extent, pa, pb, ca, s1, s2
    elif axis == 2:
        s0[0], s0[1], s0[2], s0[3], s0[4], s0[5] = pa, pb, extent, s1, s2, ca
    else:
        s0[0], s0[1], s0[2], s0[3], s0[4], s0[5] = pa, extent, pb, s1, ca, s2
    return s0
