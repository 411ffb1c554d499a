"""ctypes binding of the C ABI declared in include/mbm_b200.h.

The shared library is built in place by ``multiblockmomentsfv_b200.build``.  There
is no fallback: if the library is missing or a call fails, a ``MBMError`` is raised.
"""
from __future__ import annotations

import ctypes as C
import os

from . import build as _build

MBM_OK, MBM_EINVAL, MBM_ENONFINITE, MBM_ETIMEOUT, MBM_ECUDA, MBM_ENOMEM, MBM_ESTEPLIMIT, MBM_ENODEV = range(8)
L_DATA, L_TMP, L_NEW = 0, 1, 2
MODE_EXACT = 0
MODE_FAST = 1
MODES = {"exact": MODE_EXACT, "fast": MODE_FAST}

# every symbol include/mbm_b200.h declares
EXPORTS = (
    "mbm_create", "mbm_destroy", "mbm_upload", "mbm_download", "mbm_set_dirichlet",
    "mbm_set_boundary", "mbm_update", "mbm_time_update", "mbm_steps", "mbm_steps_capped",
    "mbm_time_stage", "mbm_trace", "mbm_attempts", "mbm_case_status", "mbm_config",
    "mbm_create_batch", "mbm_steps_batch", "mbm_trace_case", "mbm_stage_noalloc", "mbm_bulk_copies", "mbm_load_fields", "mbm_config_stage", "mbm_ghost_scatter", "mbm_dependent_launch", "mbm_set_functional",
    "mbm_adjoint_run", "mbm_replay", "mbm_set_physics", "mbm_output_fields",
    "mbm_ghost_map", "mbm_strerror", "mbm_last_error", "mbm_version",
    "mbm_shard_plan", "mbm_create_sharded", "mbm_shard_buffers", "mbm_shard_set_dirichlet",
    "mbm_shard_begin", "mbm_shard_stage",
    "mbm_shard_pack", "mbm_shard_fill", "mbm_shard_cfl", "mbm_shard_control", "mbm_shard_end",
    "mbm_fastmath_check", "mbm_steps_batch_async", "mbm_steps_batch_wait", "mbm_output_fields_async",
    "mbm_output_wait", "mbm_host_alloc", "mbm_host_free",
)


class BlockDesc(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("x0", C.c_double), ("y0", C.c_double),
                ("dx", C.c_double), ("dy", C.c_double), ("bc", C.c_int * 4)]


class Params(C.Structure):
    _fields_ = [("Kn", C.c_double), ("F", C.c_double), ("limiter", C.c_int), ("mode", C.c_int),
                ("device", C.c_int), ("show_every", C.c_int), ("max_attempts", C.c_int),
                ("segment_rows", C.c_int), ("stream", C.c_void_p), ("adjoint", C.c_int)]


class CaseDesc(C.Structure):
    _fields_ = [("first_block", C.c_int), ("nblocks", C.c_int), ("Kn", C.c_double), ("F", C.c_double),
                ("limiter", C.c_int)]


class MBMError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{msg} (status {status})")
        self.status = status


_lib = None


def lib(path: str = None):
    """Load the library (building it first if it is missing).  MBM_LIBRARY may name
    another build of it (e.g. a variant under test)."""
    global _lib
    if _lib is not None:
        return _lib
    if path is None:
        path = os.environ.get("MBM_LIBRARY") or _build.LIB
        if not os.path.exists(path):
            _build.build()
    L = C.CDLL(path)
    P = C.POINTER
    dp = P(C.c_double)
    vp = C.c_void_p
    L.mbm_create.argtypes = [P(BlockDesc), C.c_int, P(Params), P(vp)]
    L.mbm_destroy.argtypes = [vp]
    L.mbm_upload.argtypes = [vp, C.c_int, C.c_int, dp]
    L.mbm_download.argtypes = [vp, C.c_int, C.c_int, dp]
    L.mbm_set_dirichlet.argtypes = [vp, C.c_int, C.c_int, dp]
    L.mbm_set_boundary.argtypes = [vp, C.c_int, C.c_double]
    L.mbm_update.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, dp]
    L.mbm_time_update.argtypes = [vp, C.c_double, C.c_double, dp]
    L.mbm_steps.argtypes = [vp, dp, C.c_double, C.c_double, C.c_double, P(C.c_int), P(C.c_int)]
    L.mbm_steps_capped.argtypes = [vp, dp, C.c_double, C.c_double, C.c_double, C.c_int, P(C.c_int),
                                   P(C.c_int)]
    L.mbm_time_stage.argtypes = [vp, C.c_int, C.c_double, C.c_int, dp]
    L.mbm_trace.argtypes = [vp, dp, C.c_int, P(C.c_int)]
    L.mbm_attempts.argtypes = [vp, P(C.c_int)]
    L.mbm_case_status.argtypes = [vp, P(C.c_int), C.c_int]
    ip = P(C.c_int)
    L.mbm_shard_plan.argtypes = [P(BlockDesc), C.c_int, ip, C.c_int, C.c_int, ip, ip, ip, ip, C.c_int]
    L.mbm_create_sharded.argtypes = [P(BlockDesc), C.c_int, ip, C.c_int, C.c_int, P(Params), P(vp)]
    L.mbm_shard_buffers.argtypes = [vp, ip, ip, C.c_int, P(vp), P(vp), P(vp)]
    L.mbm_shard_set_dirichlet.argtypes = [vp, C.c_int, C.c_int, dp]
    L.mbm_shard_begin.argtypes = [vp, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int]
    L.mbm_shard_stage.argtypes = [vp, C.c_int]
    L.mbm_shard_pack.argtypes = [vp, C.c_int]
    L.mbm_shard_fill.argtypes = [vp, C.c_int]
    L.mbm_shard_cfl.argtypes = [vp]
    L.mbm_shard_control.argtypes = [vp, ip]
    L.mbm_shard_end.argtypes = [vp, dp, ip, ip]
    L.mbm_fastmath_check.argtypes = [vp, C.c_int, vp]
    L.mbm_steps_batch_async.argtypes = [vp, dp, dp, C.c_double, C.c_double, C.c_int]
    L.mbm_steps_batch_wait.argtypes = [vp, dp, ip, ip]
    L.mbm_output_fields_async.argtypes = [vp, C.c_int, C.c_int, vp]
    L.mbm_output_wait.argtypes = [vp]
    L.mbm_host_alloc.argtypes = [C.c_size_t, P(vp)]
    L.mbm_host_free.argtypes = [vp]
    L.mbm_config.argtypes = [vp, P(C.c_int), P(C.c_int), P(C.c_int)]
    L.mbm_create_batch.argtypes = [P(BlockDesc), C.c_int, P(CaseDesc), C.c_int, P(Params), P(vp)]
    L.mbm_steps_batch.argtypes = [vp, dp, dp, C.c_double, C.c_double, C.c_int, P(C.c_int), P(C.c_int)]
    L.mbm_trace_case.argtypes = [vp, C.c_int, dp, C.c_int, P(C.c_int)]
    L.mbm_adjoint_run.argtypes = [vp, dp, C.c_int, C.c_int, C.c_double, dp, dp, dp, dp, dp]
    L.mbm_replay.argtypes = [vp, dp, C.c_int, dp]
    L.mbm_set_physics.argtypes = [vp, C.c_double, C.c_double]
    L.mbm_set_functional.argtypes = [vp, C.c_int]
    L.mbm_dependent_launch.argtypes = [vp, P(C.c_int)]
    L.mbm_ghost_scatter.argtypes = [vp, P(C.c_int)]
    L.mbm_config_stage.argtypes = [vp, C.c_int, dp, P(C.c_int), P(C.c_int)]
    L.mbm_load_fields.argtypes = [vp, C.c_int, C.c_int, vp, C.c_int]
    L.mbm_output_fields.argtypes = [vp, C.c_int, C.c_int, vp]
    L.mbm_bulk_copies.argtypes = [vp, P(C.c_int)]
    L.mbm_stage_noalloc.argtypes = [P(BlockDesc), C.c_int, vp, vp, vp, C.c_double, C.c_double, C.c_int,
                                    C.c_double, C.c_int, dp, vp]
    L.mbm_ghost_map.argtypes = [P(BlockDesc), C.c_int, P(C.c_int), C.c_int, P(C.c_int)]
    L.mbm_strerror.restype = C.c_char_p
    L.mbm_strerror.argtypes = [C.c_int]
    L.mbm_last_error.restype = C.c_char_p
    L.mbm_last_error.argtypes = [vp]
    for name in EXPORTS:
        getattr(L, name).restype = getattr(L, name).restype or C.c_int
    L.mbm_strerror.restype = C.c_char_p
    L.mbm_last_error.restype = C.c_char_p
    _lib = L
    return L


def check(status: int, ctx=None) -> None:
    if status != MBM_OK:
        L = lib()
        msg = L.mbm_last_error(ctx).decode() or L.mbm_strerror(status).decode()
        raise MBMError(status, msg)


def block_descs(blocks):
    arr = (BlockDesc * len(blocks))()
    for i, b in enumerate(blocks):
        arr[i].nx, arr[i].ny = b.nx, b.ny
        arr[i].x0, arr[i].y0, arr[i].dx, arr[i].dy = b.x0, b.y0, b.dx, b.dy
        for s in range(4):
            arr[i].bc[s] = b.bc[s]
    return arr
