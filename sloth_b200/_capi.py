"""ctypes binding of ``libsloth_b200.so`` (declared in ``include/sloth_b200.h``).

The library is the only compute path of this package: there is no CPU or
PyTorch fallback. If the shared object is missing the import of this module
raises ``SlothExtensionMissing``; if there is no usable sm_100 device, the
compute entry points return ``SLOTH_ERR_NO_DEVICE`` /
``SLOTH_ERR_UNSUPPORTED_DEVICE`` and ``check`` raises ``SlothError``.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import (POINTER, Structure, c_char_p, c_double, c_int, c_int32, c_int64,
                    c_size_t, c_uint8, c_ulonglong, c_void_p)

_HERE = os.path.dirname(os.path.abspath(__file__))
# SLOTH_B200_LIB selects another build of the same library (e.g. a tuning variant).
LIB_PATH = os.environ.get("SLOTH_B200_LIB") or os.path.join(_HERE, "_lib", "libsloth_b200.so")

SLOTH_OK = 0
SLOTH_ERR_INVALID_ARGUMENT = -1
SLOTH_ERR_NULL_POINTER = -2
SLOTH_ERR_MISALIGNED = -3
SLOTH_ERR_WORKSPACE_TOO_SMALL = -4
SLOTH_ERR_CUDA = -5
SLOTH_ERR_NO_DEVICE = -6
SLOTH_ERR_TOO_LARGE = -7
SLOTH_ERR_OUT_OF_MEMORY = -8
SLOTH_ERR_NOT_FOUND = -9
SLOTH_ERR_BUSY = -10
SLOTH_ERR_UNSUPPORTED_DEVICE = -11

SLOTH_RAY_EXITED = 0
SLOTH_RAY_INSIDE_AT_END = 1
SLOTH_RAY_NONFINITE = 2

SLOTH_MAX_SAVES = 4096
SLOTH_NOALLOC_MAX_RAYS = 1 << 20


class SlothExtensionMissing(ImportError):
    """The compiled CUDA library is not present (build it with ``make`` in csrc/)."""


class SlothError(RuntimeError):
    """A library entry point returned a negative status code."""

    def __init__(self, code: int, what: str = ""):
        self.code = code
        msg = strerror(code)
        super().__init__(f"{what}: {msg} (code {code})" if what else f"{msg} (code {code})")


class SlothGridDesc(Structure):
    _fields_ = [("n", c_int32 * 3), ("reserved", c_int32),
                ("origin", c_double * 3), ("spacing", c_double * 3)]


class SlothTraceParams(Structure):
    _fields_ = [("omega", c_double), ("dtau", c_double),
                ("first_save", c_int32), ("save_every", c_int32), ("n_saves", c_int32),
                ("probing_axis", c_int32), ("project_to_plane", c_int32), ("inv_brems", c_int32),
                ("plane", c_double), ("kappa_q2", c_double), ("coulomb_log_w", c_double),
                ("ope_ratio2", c_double), ("q_max", c_double), ("q_min", c_double),
                ("integrator", c_int32), ("reserved", c_int32)]


class SlothTraceOutputs(Structure):
    _fields_ = [("jones", c_void_p), ("state", c_void_p), ("phase", c_void_p),
                ("amp", c_void_p), ("status", c_void_p), ("steps", c_void_p),
                ("total_steps", c_void_p), ("trace_event_begin", c_void_p), ("trace_event_end", c_void_p)]


class SlothServerConfig(Structure):
    _fields_ = [("budget_bytes", c_size_t), ("max_jobs", c_int32), ("tiles_per_step", c_int32),
                ("quantum", c_int32), ("reserved", c_int32)]


class SlothServerStats(Structure):
    _fields_ = [("budget_bytes", c_size_t), ("arena_used", c_size_t), ("grids_resident", ctypes.c_longlong),
                ("grid_packs", ctypes.c_longlong), ("grid_evictions", ctypes.c_longlong),
                ("jobs_submitted", ctypes.c_longlong), ("jobs_admitted", ctypes.c_longlong),
                ("jobs_done", ctypes.c_longlong), ("jobs_failed", ctypes.c_longlong),
                ("iterations", ctypes.c_longlong), ("tiles", ctypes.c_longlong),
                ("kernel_launches", ctypes.c_longlong), ("gpu_busy_ms", c_double), ("gpu_span_ms", c_double),
                ("jobs_cancelled", ctypes.c_longlong), ("cancelled_pending_free", ctypes.c_longlong)]


class SlothOptic(Structure):
    _fields_ = [("kind", c_int32), ("axis", c_int32), ("a", c_double), ("b", c_double)]


class SlothDetectorParams(Structure):
    _fields_ = [("nx", c_int32), ("ny", c_int32), ("x_range", c_double * 2), ("y_range", c_double * 2),
                ("pos_scale", c_double), ("prefilter", c_int32), ("ccd_clip", c_int32), ("prefilter_L", c_double),
                ("prefilter_R", c_double), ("ccd_half", c_double * 2), ("reserved", c_int32),
                ("reserved2", c_int32)]


(SLOTH_OPTIC_TRAVEL, SLOTH_OPTIC_LENS, SLOTH_OPTIC_CIRCULAR_APERTURE, SLOTH_OPTIC_CIRCULAR_STOP,
 SLOTH_OPTIC_RECT_APERTURE, SLOTH_OPTIC_KNIFE_EDGE, SLOTH_OPTIC_ANNULAR_STOP) = range(1, 8)
SLOTH_MAX_OPTICS = 32


class SlothBeamParams(Structure):
    _fields_ = [("beam_type", c_int32), ("probing_axis", c_int32), ("size", c_double * 2), ("divergence", c_double),
                ("ne_extent", c_double), ("seed", ctypes.c_uint64), ("first_id", ctypes.c_uint64),
                ("reserved", c_int32), ("reserved2", c_int32)]


SLOTH_BEAM_CIRCULAR, SLOTH_BEAM_SQUARE, SLOTH_BEAM_RECTANGULAR, SLOTH_BEAM_LINEAR = 0, 1, 2, 3


class SlothImageParams(Structure):
    _fields_ = [("dtau", c_double), ("n_steps", c_int32), ("ckpt_every", c_int32), ("probing_axis", c_int32),
                ("n_px", c_int32 * 2), ("reserved", c_int32), ("plane", c_double), ("window", c_double * 4),
                ("sigma_px", c_double)]


SLOTH_JOB_PENDING, SLOTH_JOB_RUNNING, SLOTH_JOB_DONE, SLOTH_JOB_FETCHING, SLOTH_JOB_FETCHED = 0, 1, 2, 3, 4
SLOTH_JOB_CANCELLED = 5
SLOTH_INTEGRATOR_RKN, SLOTH_INTEGRATOR_RK4 = 0, 1

# name -> (restype, argtypes); every symbol include/sloth_b200.h declares.
_SIGNATURES = {
    "sloth_strerror": (c_char_p, [c_int]),
    "sloth_abi_version": (c_int, []),
    "sloth_device_info": (c_int, [POINTER(c_int), POINTER(c_int), POINTER(c_int)]),
    "sloth_launch_count": (c_ulonglong, []),
    "sloth_grid_bytes": (c_size_t, [POINTER(SlothGridDesc), c_int]),
    "sloth_grid_pack_f32": (c_int, [POINTER(SlothGridDesc), c_void_p, c_int, c_double, c_void_p, c_void_p]),
    "sloth_grid_pack_f64": (c_int, [POINTER(SlothGridDesc), c_void_p, c_int, c_double, c_void_p, c_void_p]),
    "sloth_grid_pack_trace_f32": (c_int, [POINTER(SlothGridDesc), c_void_p, c_int, c_double, c_double, c_void_p,
                                          c_void_p]),
    "sloth_grid_pack_trace_f64": (c_int, [POINTER(SlothGridDesc), c_void_p, c_int, c_double, c_double, c_void_p,
                                          c_void_p]),
    "sloth_sample_f32": (c_int, [POINTER(SlothGridDesc), c_void_p, c_void_p, c_int64, c_void_p, c_void_p]),
    "sloth_sample_f64": (c_int, [POINTER(SlothGridDesc), c_void_p, c_void_p, c_int64, c_void_p, c_void_p]),
    "sloth_trace_workspace_bytes": (c_size_t, [c_int64]),
    "sloth_trace_f32": (c_int, [POINTER(SlothGridDesc), c_void_p, POINTER(SlothTraceParams), c_void_p,
                                c_int64, POINTER(SlothTraceOutputs), c_void_p, c_size_t, c_void_p]),
    "sloth_trace_f64": (c_int, [POINTER(SlothGridDesc), c_void_p, POINTER(SlothTraceParams), c_void_p,
                                c_int64, POINTER(SlothTraceOutputs), c_void_p, c_size_t, c_void_p]),
    "sloth_trace_f32_noalloc": (c_int, [POINTER(SlothGridDesc), c_void_p, POINTER(SlothTraceParams), c_void_p,
                                        c_int64, POINTER(SlothTraceOutputs), c_void_p]),
    "sloth_server_create": (c_int, [POINTER(SlothServerConfig), POINTER(c_void_p)]),
    "sloth_server_destroy": (c_int, [c_void_p]),
    "sloth_server_submit": (c_int, [c_void_p, ctypes.c_uint64, POINTER(SlothGridDesc), c_void_p, c_int,
                                    POINTER(SlothTraceParams), c_void_p, c_int, c_int64, POINTER(c_int)]),
    "sloth_server_step": (c_int, [c_void_p, POINTER(c_int), POINTER(c_int)]),
    "sloth_server_job_state": (c_int, [c_void_p, c_int, POINTER(c_int)]),
    "sloth_server_fetch": (c_int, [c_void_p, c_int, POINTER(SlothTraceOutputs)]),
    "sloth_server_release": (c_int, [c_void_p, c_int]),
    "sloth_server_stats": (c_int, [c_void_p, POINTER(SlothServerStats)]),
    "sloth_server_sync": (c_int, [c_void_p]),
    "sloth_server_cancel": (c_int, [c_void_p, c_int]),
    "sloth_server_inject_alloc_failure": (c_int, [c_int]),
    "sloth_image_workspace_bytes": (c_size_t, [POINTER(SlothImageParams), c_int64]),
    "sloth_image_forward_f32": (c_int, [POINTER(SlothGridDesc), c_void_p, POINTER(SlothImageParams), c_void_p,
                                        c_int64, c_void_p, c_void_p, c_void_p, c_size_t, c_void_p]),
    "sloth_image_forward_f64": (c_int, [POINTER(SlothGridDesc), c_void_p, POINTER(SlothImageParams), c_void_p,
                                        c_int64, c_void_p, c_void_p, c_void_p, c_size_t, c_void_p]),
    "sloth_image_backward_f32": (c_int, [POINTER(SlothGridDesc), c_void_p, POINTER(SlothImageParams), c_int64,
                                         c_void_p, c_void_p, c_void_p, c_size_t, c_void_p]),
    "sloth_image_backward_f64": (c_int, [POINTER(SlothGridDesc), c_void_p, POINTER(SlothImageParams), c_int64,
                                         c_void_p, c_void_p, c_void_p, c_size_t, c_void_p]),
    "sloth_grid_pack_adjoint_f32": (c_int, [POINTER(SlothGridDesc), c_void_p, c_double, c_void_p, c_void_p]),
    "sloth_grid_pack_adjoint_f64": (c_int, [POINTER(SlothGridDesc), c_void_p, c_double, c_void_p, c_void_p]),
    "sloth_optics_f32": (c_int, [c_void_p, c_int64, c_void_p, POINTER(SlothOptic), c_int32,
                                 POINTER(SlothDetectorParams), c_void_p, c_void_p, c_void_p, c_void_p]),
    "sloth_optics_f64": (c_int, [c_void_p, c_int64, c_void_p, POINTER(SlothOptic), c_int32,
                                 POINTER(SlothDetectorParams), c_void_p, c_void_p, c_void_p, c_void_p]),
    "sloth_beam_f32": (c_int, [POINTER(SlothBeamParams), c_int64, c_void_p, c_void_p]),
    "sloth_beam_f64": (c_int, [POINTER(SlothBeamParams), c_int64, c_void_p, c_void_p]),
}

EXPORTED_SYMBOLS = tuple(_SIGNATURES)

_lib = None


def load() -> ctypes.CDLL:
    """Load the library once; raise SlothExtensionMissing if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise SlothExtensionMissing(
            f"{LIB_PATH} not found: build it with `make -C {os.path.join(_HERE, 'csrc')}` "
            "(or __graft_entry__.build()); there is no fallback implementation")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def strerror(code: int) -> str:
    try:
        return load().sloth_strerror(int(code)).decode()
    except SlothExtensionMissing:
        return f"error {code}"


def check(rc: int, what: str = "") -> None:
    if rc != SLOTH_OK:
        raise SlothError(rc, what)


def launch_count() -> int:
    return int(load().sloth_launch_count())


def device_info():
    sms, ma, mi = c_int(0), c_int(0), c_int(0)
    check(load().sloth_device_info(ctypes.byref(sms), ctypes.byref(ma), ctypes.byref(mi)), "sloth_device_info")
    return sms.value, ma.value, mi.value


def grid_desc(n, origin, spacing) -> SlothGridDesc:
    g = SlothGridDesc()
    for a in range(3):
        g.n[a] = int(n[a])
        g.origin[a] = float(origin[a])
        g.spacing[a] = float(spacing[a])
    g.reserved = 0
    return g


def ptr(t) -> int:
    """Device pointer of a torch tensor (or 0 for None)."""
    return 0 if t is None else int(t.data_ptr())
