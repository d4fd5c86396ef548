"""ctypes binding of ``include/mun_sem.h`` (the library is ``mun_b200/_sem.so``).

There is no CPU fallback: if the library is missing or fails to load, every entry
point raises ``RuntimeError``.
"""
import ctypes as C
import os

from . import build as _build

_HERE = os.path.dirname(os.path.abspath(__file__))

SEM_OK, SEM_ERR_ARG, SEM_ERR_CUDA, SEM_ERR_OOM, SEM_ERR_NONFINITE, SEM_ERR_TIMEOUT, \
    SEM_ERR_UNSUPPORTED = range(7)
SEM_F_ADJOINT, SEM_F_EXACT, SEM_F_MISFIT, SEM_F_SHIFT = 1, 2, 4, 8


class PlanDesc(C.Structure):
    _fields_ = [("nelx", C.c_int32), ("nelz", C.c_int32), ("npol", C.c_int32), ("nt", C.c_int32),
                ("npoints", C.c_int32), ("dt", C.c_double),
                ("node_grid", C.POINTER(C.c_int64)), ("gll_D", C.POINTER(C.c_double)),
                ("gll_beta", C.POINTER(C.c_double)), ("tab_x", C.POINTER(C.c_double)),
                ("tab_z", C.POINTER(C.c_double)), ("src_term", C.POINTER(C.c_double)),
                ("src_gx", C.c_int32), ("src_gz", C.c_int32), ("nrec", C.c_int32),
                ("rec_base", C.POINTER(C.c_int32)), ("rec_w", C.POINTER(C.c_double)),
                ("boundary_mode", C.c_int32), ("bnd_n", C.c_int32), ("bnd_ref", C.POINTER(C.c_int32)),
                ("bnd_alpha", C.POINTER(C.c_double)), ("bnd_gamma", C.POINTER(C.c_double))]


class Solve(C.Structure):
    _fields_ = [("plan", C.c_void_p), ("velocity", C.c_void_p), ("flags", C.c_int32),
                ("ckpt_k", C.c_int32), ("y_obs", C.c_void_p), ("it0", C.c_int32),
                ("it1", C.c_int32), ("decim", C.c_int32), ("inv_sigma2", C.c_double),
                ("rec_out", C.c_void_p), ("loglik_out", C.c_void_p), ("grad_out", C.c_void_p),
                ("status_out", C.c_void_p)]


class LaunchCfg(C.Structure):
    _fields_ = [("tile_ex", C.c_int32), ("tile_ez", C.c_int32), ("threads", C.c_int32),
                ("graph_chunk", C.c_int32), ("kernel", C.c_int32), ("strip_bands", C.c_int32),
                ("memory_budget", C.c_int64)]


class CurveDesc(C.Structure):
    _fields_ = [("ncoef", C.c_int32), ("knots", C.POINTER(C.c_double)), ("coef", C.POINTER(C.c_double)),
                ("u_lo", C.c_double), ("u_hi", C.c_double), ("nsamples", C.c_int32),
                ("u0", C.c_void_p), ("samples", C.c_void_p), ("newton_steps", C.c_int32),
                ("tau", C.c_double), ("v_inside", C.c_double), ("blend_replace", C.c_int32)]


class EngineCfg(C.Structure):
    _fields_ = [("max_solves", C.c_int32), ("memory_cap", C.c_int64), ("ticks_per_step", C.c_int32),
                ("kernel", C.c_int32), ("tile_ex", C.c_int32), ("tile_ez", C.c_int32)]


EXPORTS = ["sem_plan_create", "sem_plan_destroy", "sem_plan_workspace_bytes", "sem_batch_create",
           "sem_batch_destroy", "sem_run", "sem_batch_last_launches", "sem_batch_last_kernel",
           "sem_batch_last_groups", "sem_batch_last_shape", "sem_batch_last_ticks",
           "sem_batch_last_tick_ms", "sem_forward",
           "sem_forward_adjoint", "sem_forward_noalloc", "sem_selftest_wait", "sem_engine_create", "sem_engine_destroy",
           "sem_engine_submit", "sem_engine_step", "sem_engine_status", "sem_engine_release",
           "sem_engine_stats", "sem_velocity_from_curve", "sem_project_from_curve",
           "sem_velocity_last_error", "sem_last_error"]

_lib = None


def load(path=None):
    """Load (building first if the sources are newer and nvcc exists) the library."""
    global _lib
    if _lib is not None:
        return _lib
    so = path or os.path.join(_HERE, "_sem.so")
    if path is None:
        try:
            if _build.needs_build():
                _build.build()
        except Exception as exc:  # no nvcc: use what is there, or fail below
            if not os.path.exists(so):
                raise RuntimeError(f"mun_b200 CUDA library missing and cannot be built: {exc}")
    if not os.path.exists(so):
        raise RuntimeError(f"mun_b200 CUDA library not found at {so}")
    lib = C.CDLL(so)
    vp, i32, i64, dbl = C.c_void_p, C.c_int32, C.c_int64, C.c_double
    lib.sem_plan_create.argtypes = [C.POINTER(PlanDesc), C.POINTER(vp)]
    lib.sem_plan_destroy.argtypes = [vp]
    lib.sem_plan_workspace_bytes.argtypes = [vp, i32, i32]
    lib.sem_plan_workspace_bytes.restype = i64
    lib.sem_batch_create.argtypes = [C.POINTER(vp)]
    lib.sem_batch_destroy.argtypes = [vp]
    lib.sem_run.argtypes = [vp, C.POINTER(Solve), i32, C.POINTER(LaunchCfg), vp]
    lib.sem_batch_last_launches.argtypes = [vp]
    lib.sem_batch_last_launches.restype = i64
    lib.sem_batch_last_kernel.argtypes = [vp]
    lib.sem_batch_last_kernel.restype = i32
    lib.sem_batch_last_groups.argtypes = [vp]
    lib.sem_batch_last_groups.restype = i32
    lib.sem_batch_last_shape.argtypes = [vp, vp, vp, vp]
    lib.sem_batch_last_ticks.argtypes = [vp]
    lib.sem_batch_last_ticks.restype = i64
    lib.sem_batch_last_tick_ms.argtypes = [vp, C.POINTER(C.c_double)]
    lib.sem_forward.argtypes = [vp, vp, vp, vp, vp]
    lib.sem_forward_adjoint.argtypes = [vp, vp, vp, vp, dbl, i32, i32, vp, vp, vp, vp]
    lib.sem_forward_noalloc.argtypes = [vp, vp, vp, vp, vp]
    lib.sem_selftest_wait.argtypes = [i32, vp]
    lib.sem_engine_create.argtypes = [C.POINTER(EngineCfg), C.POINTER(vp)]
    lib.sem_engine_destroy.argtypes = [vp]
    lib.sem_engine_submit.argtypes = [vp, C.POINTER(Solve), C.POINTER(i64)]
    lib.sem_engine_step.argtypes = [vp, vp]
    lib.sem_engine_status.argtypes = [vp, i64, C.POINTER(i32)]
    lib.sem_engine_release.argtypes = [vp, i64]
    lib.sem_engine_stats.argtypes = [vp, C.POINTER(i64)]
    lib.sem_velocity_from_curve.argtypes = [C.POINTER(CurveDesc), i32, vp, vp, dbl, vp, vp, vp, vp, vp]
    lib.sem_project_from_curve.argtypes = [vp, i32, i32, i32, i32, i32, vp, vp, vp, vp, vp, dbl, dbl,
                                           dbl, i32, vp, vp]
    lib.sem_velocity_last_error.restype = C.c_char_p
    lib.sem_last_error.restype = C.c_char_p
    for name in EXPORTS:
        if name not in ("sem_plan_workspace_bytes", "sem_batch_last_launches", "sem_batch_last_kernel",
                        "sem_batch_last_groups", "sem_batch_last_ticks", "sem_last_error", "sem_velocity_last_error"):
            getattr(lib, name).restype = C.c_int
    _lib = lib
    return lib


def check(code):
    if code == SEM_OK:
        return
    msg = load().sem_last_error().decode(errors="replace")
    if code == SEM_ERR_ARG or code == SEM_ERR_UNSUPPORTED:
        raise ValueError(f"mun_b200: {msg}")
    if code == SEM_ERR_OOM:
        raise MemoryError(f"mun_b200: {msg}")
    raise RuntimeError(f"mun_b200 (status {code}): {msg}")
