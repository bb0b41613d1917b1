"""ctypes declarations of the trace entry points of sloth_b200.h.

This is the binding a SLOTH maintainer adds beside src/core/propagator.py:
SLOTH is pure Python, so its foreign-function interface is ctypes. It takes
device pointers from any framework that exposes them (torch ``data_ptr()``,
CuPy, DLPack) and declares only what a trace needs: the grid pack (K1, trace layout), the
workspace size, the FP32 / FP64 tracers and the error text. The structs
mirror ``SlothGridDesc``, ``SlothTraceParams`` and ``SlothTraceOutputs`` field
for field; the package's own binding (sloth_b200/_capi.py) covers the whole
header.

In ``solve()`` the block ``jax.vmap(ODE_solve, in_axes=(0, None))(s0, args)``
(src/core/propagator.py:785-793) and ``process_results`` (:926) become one
``sloth_trace_f32`` call with ``n_saves = save_points_per_region``; in
``trace_and_save_depths`` the vmapped solve and the per-save
``ray_to_Jonesvector`` loop (:1196-1218) become one call with
``first_save = 0`` and ``save_every`` = the steps of one depth step.
"""
import ctypes
from ctypes import POINTER, Structure, c_double, c_int, c_int32, c_int64, c_size_t, c_void_p


class GridDesc(Structure):
    _fields_ = [("n", c_int32 * 3), ("reserved", c_int32), ("origin", c_double * 3), ("spacing", c_double * 3)]


class TraceParams(Structure):
    _fields_ = [("omega", c_double), ("dtau", c_double), ("first_save", c_int32), ("save_every", c_int32),
                ("n_saves", c_int32), ("probing_axis", c_int32), ("project_to_plane", c_int32),
                ("inv_brems", c_int32), ("plane", c_double), ("kappa_q2", c_double),
                ("coulomb_log_w", c_double), ("ope_ratio2", c_double), ("q_max", c_double),
                ("q_min", c_double), ("integrator", c_int32), ("reserved", c_int32)]


class TraceOutputs(Structure):
    _fields_ = [(k, c_void_p) for k in ("jones", "state", "phase", "amp", "status", "steps",
                                        "total_steps", "trace_event_begin", "trace_event_end")]


def load(path="libsloth_b200.so"):
    """Opens the library and declares the trace entry points' signatures."""
    lib = ctypes.CDLL(path)
    lib.sloth_grid_pack_trace_f32.restype = c_int
    lib.sloth_grid_pack_trace_f32.argtypes = [POINTER(GridDesc), c_void_p, c_int, c_double, c_double, c_void_p,
                                              c_void_p]
    lib.sloth_trace_workspace_bytes.restype = c_size_t
    lib.sloth_trace_workspace_bytes.argtypes = [c_int64]
    for name in ("sloth_trace_f32", "sloth_trace_f64"):
        fn = getattr(lib, name)
        fn.restype = c_int
        fn.argtypes = [POINTER(GridDesc), c_void_p, POINTER(TraceParams), c_void_p, c_int64,
                       POINTER(TraceOutputs), c_void_p, c_size_t, c_void_p]
    lib.sloth_strerror.restype = ctypes.c_char_p
    lib.sloth_strerror.argtypes = [c_int]
    return lib
