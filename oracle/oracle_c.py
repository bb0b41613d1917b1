"""ctypes loader of the oracle's C restatement (oracle/cpu_rk4.c).

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py). Wraps oracle_trace() with
the same inputs and outputs as ref_restated.trace_rays().
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, Structure, c_double, c_int, c_int32, c_int64, c_longlong, c_void_p

import numpy as np

from . import ref_restated as rr

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "_build", "liboracle_rk4.so")


class OracleParams(Structure):
    _fields_ = [("n", c_int32 * 3), ("pad", c_int32), ("origin", c_double * 3), ("spacing", c_double * 3),
                ("fields", c_void_p), ("kappa", c_void_p), ("omega", c_double), ("dt", c_double),
                ("first_save", c_int32), ("save_every", c_int32), ("n_saves", c_int32),
                ("axis", c_int32), ("project", c_int32), ("inv_brems", c_int32), ("early_exit", c_int32),
                ("threads", c_int32), ("plane", c_double), ("integrator", c_int32), ("pad2", c_int32),
                ("nm1", c_void_p)]


_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return LIB


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        lib = ctypes.CDLL(LIB)
        lib.oracle_trace.restype = c_int
        lib.oracle_trace.argtypes = [POINTER(OracleParams), c_void_p, c_int64, c_void_p, c_void_p,
                                     c_void_p, c_void_p, c_void_p, c_void_p, POINTER(c_longlong)]
        lib.oracle_threads.restype = c_int
        _lib = lib
    return _lib


def threads() -> int:
    return int(load().oracle_threads())


def trace_rays(grid: "rr.Grid", rays, *, dtau, first_save, save_every, n_saves, axis=2, project=False,
               plane=0.0, inv_brems=False, early_exit=True, threads=0, want_state=True, integrator="rkn"):
    """C version of ref_restated.trace_rays (phase_mode 'reference': the
    interpolated n - 1 grid); integrator 'rkn' (Runge-Kutta-Nystrom, 3
    samples) or 'rk4' (classical RK4, 4)."""
    lib = load()
    rays = np.ascontiguousarray(rays, dtype=np.float64)
    n = rays.shape[1]
    fields = np.ascontiguousarray(grid.fields, dtype=np.float64)
    kappa = None
    if inv_brems:
        kappa = np.ascontiguousarray(grid.kappa, dtype=np.float64)
    p = OracleParams()
    for a in range(3):
        p.n[a] = grid.n[a]
        p.origin[a] = grid.origin[a]
        p.spacing[a] = grid.spacing[a]
    p.fields = fields.ctypes.data
    nm1 = np.ascontiguousarray(grid.nm1, dtype=np.float64)
    p.nm1 = nm1.ctypes.data
    p.kappa = kappa.ctypes.data if kappa is not None else None
    p.omega = grid.omega
    p.dt = dtau / rr.C
    p.first_save, p.save_every, p.n_saves = first_save, save_every, n_saves
    p.axis, p.project, p.inv_brems, p.early_exit = axis, int(project), int(inv_brems), int(early_exit)
    p.threads = threads
    p.plane = plane
    p.integrator = {"rkn": 0, "rk4": 1}[integrator]
    S = n_saves
    state = np.zeros((S, 6, n)) if want_state else None
    jones = np.zeros((S, 4, n))
    phase = np.zeros((S, n))
    tau = np.zeros((S, n))
    steps = np.zeros(n, dtype=np.int32)
    status = np.zeros(n, dtype=np.uint8)
    tot = c_longlong(0)
    rc = lib.oracle_trace(ctypes.byref(p), rays.ctypes.data, n,
                          state.ctypes.data if state is not None else None, jones.ctypes.data,
                          phase.ctypes.data, tau.ctypes.data, steps.ctypes.data, status.ctypes.data,
                          ctypes.byref(tot))
    if rc != 0:
        raise RuntimeError(f"oracle_trace failed ({rc})")
    return dict(state=state, jones=jones, phase=phase, tau=tau, amp=np.exp(-tau), steps=steps,
                status=status, total_steps=int(tot.value))
