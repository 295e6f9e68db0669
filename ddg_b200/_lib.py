"""ctypes binding of ``libddg_sipg.so`` (the C ABI in ``include/ddg_sipg.h``).

The library is built in-tree (``python -m ddg_b200.build``).  There is no
fallback: if the shared library is missing or a GPU entry point fails, a
``DdgError`` is raised.
"""

from __future__ import annotations

import ctypes as C
import os

from .build import LIB as _LIB_PATH

DDG_OK = 0
DDG_FP64 = 0
DDG_FP32 = 1
DDG_PC_NONE = 0
DDG_PC_JACOBI = 1
DDG_MAX_DEGREE = 5
DDG_ENGINE_CUDA_CORES = 0
DDG_ENGINE_TENSOR_CORES = 1
DDG_QUAD_NODAL = 0
DDG_QUAD_CUBATURE = 1
SOLVE_STATUS = {0: "converged", 1: "maxiter", 2: "breakdown", 3: "device_error", 4: "stagnated"}


class DdgError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, code: int, where: str, msg: str):
        super().__init__(f"{where} failed (status {code}): {msg}")
        self.code = code


class MeshDesc(C.Structure):
    _fields_ = [("N", C.c_int32), ("K", C.c_int32), ("device", C.c_int32), ("reserved", C.c_int32),
                ("tau_scale", C.c_double),
                ("Dr", C.POINTER(C.c_double)), ("Ds", C.POINTER(C.c_double)),
                ("M", C.POINTER(C.c_double)), ("m1d", C.POINTER(C.c_double)),
                ("Fmask", C.POINTER(C.c_int64)), ("rot_perm", C.POINTER(C.c_int64)),
                ("geo", C.POINTER(C.c_double)),
                ("EToE", C.POINTER(C.c_int64)), ("EToF", C.POINTER(C.c_int64)),
                ("vmapM", C.POINTER(C.c_int64)), ("vmapP", C.POINTER(C.c_int64)),
                ("bc_types", C.POINTER(C.c_int32))]


_dp = C.POINTER(C.c_double)


class CurvedDesc(C.Structure):
    _fields_ = [("N", C.c_int32), ("K", C.c_int32), ("device", C.c_int32), ("Ncub", C.c_int32),
                ("Nfq", C.c_int32), ("reserved", C.c_int32), ("tau_scale", C.c_double),
                ("Dr", _dp), ("Ds", _dp), ("M", _dp), ("m1d", _dp), ("Fmask", C.POINTER(C.c_int64)),
                ("rx", _dp), ("sx", _dp), ("ry", _dp), ("sy", _dp), ("J", _dp),
                ("nx", _dp), ("ny", _dp), ("sJ", _dp), ("Fscale", _dp),
                ("EToE", C.POINTER(C.c_int64)), ("EToF", C.POINTER(C.c_int64)),
                ("vmapM", C.POINTER(C.c_int64)), ("vmapP", C.POINTER(C.c_int64)),
                ("bc_types", C.POINTER(C.c_int32)),
                ("cw", _dp), ("Drq", _dp), ("Dsq", _dp), ("Lq", _dp),
                ("cJ", _dp), ("crx", _dp), ("csx", _dp), ("cry", _dp), ("csy", _dp),
                ("face_w", _dp), ("face_L1d", _dp), ("face_sJ", _dp)]


class CgConfig(C.Structure):
    _fields_ = [("tol", C.c_double), ("atol", C.c_double), ("maxiter", C.c_int32), ("pc", C.c_int32),
                ("alpha", C.c_double), ("shift", C.c_double), ("precision", C.c_int32),
                ("reserved", C.c_int32)]


class SolveInfo(C.Structure):
    _fields_ = [("status", C.c_int32), ("iterations", C.c_int32), ("res_norm2", C.c_double),
                ("b_norm2", C.c_double), ("updates", C.c_int32), ("reserved", C.c_int32)]


class MgDesc(C.Structure):
    _fields_ = [("nlevels", C.c_int32), ("precision", C.c_int32), ("nu", C.c_int32), ("reserved", C.c_int32),
                ("omega", C.c_double), ("alpha", C.c_double),
                ("ops", C.POINTER(C.c_void_p)),
                ("prolong", C.POINTER(C.POINTER(C.c_double))),
                ("prolong_rows", C.POINTER(C.c_int32)), ("prolong_cols", C.POINTER(C.c_int32)),
                ("coarse_inv", C.POINTER(C.c_double))]


_vp = C.c_void_p
_i64 = C.c_int64
_PROTOS = {
    "ddg_sipg_create": (C.c_int, [C.POINTER(MeshDesc), C.POINTER(_vp)]),
    "ddg_sipg_destroy": (C.c_int, [_vp]),
    "ddg_sipg_set_bc": (C.c_int, [_vp, C.POINTER(C.c_int32)]),
    "ddg_sipg_apply": (C.c_int, [_vp, C.c_int, C.c_double, _vp, _vp, _vp]),
    "ddg_sipg_apply_host": (C.c_int, [_vp, C.c_double, _vp, _vp, _vp]),
    "ddg_sipg_set_engine": (C.c_int, [_vp, C.c_int]),
    "ddg_sipg_rhs": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "ddg_sipg_pc_build": (C.c_int, [_vp, C.c_double, _vp]),
    "ddg_sipg_pc_apply": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp]),
    "ddg_sipg_pc_blocks": (C.c_int, [_vp, _vp, _vp]),
    "ddg_sipg_cg": (C.c_int, [_vp, C.POINTER(CgConfig), _vp, _vp, _vp, C.POINTER(SolveInfo)]),
    "ddg_sipg_cg_mixed": (C.c_int, [_vp, C.POINTER(CgConfig), C.c_double, _vp, _vp, _vp, C.POINTER(SolveInfo)]),
    "ddg_mg_create": (C.c_int, [C.POINTER(MgDesc), C.POINTER(_vp)]),
    "ddg_mg_destroy": (C.c_int, [_vp]),
    "ddg_mg_apply": (C.c_int, [_vp, _vp, _vp, _vp]),
    "ddg_sipg_cg_mg": (C.c_int, [_vp, C.POINTER(CgConfig), _vp, _vp, _vp, _vp, C.POINTER(SolveInfo)]),
    "ddg_pool_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.POINTER(_vp)]),
    "ddg_pool_create_ex": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int,
                                     C.POINTER(_vp)]),
    "ddg_pool_destroy": (C.c_int, [_vp]),
    "ddg_pool_admit": (C.c_int, [_vp, C.POINTER(MeshDesc), C.c_double, C.c_double, C.c_double, C.c_int, _vp, _vp,
                                 C.POINTER(C.c_int)]),
    "ddg_pool_iterate": (C.c_int, [_vp, C.c_int, _vp]),
    "ddg_pool_set_tile": (C.c_int, [_vp, C.c_int, C.c_int]),
    "ddg_pool_poll": (C.c_int, [_vp, _vp, _vp, _vp]),
    "ddg_pool_retire": (C.c_int, [_vp, C.c_int, _vp, _vp, C.POINTER(SolveInfo)]),
    "ddg_sipg_upload_reference": (C.c_int, [C.c_int, _vp, _vp, _vp, _vp, C.c_int]),
    "ddg_curved_create": (C.c_int, [C.POINTER(CurvedDesc), C.POINTER(_vp)]),
    "ddg_curved_destroy": (C.c_int, [_vp]),
    "ddg_curved_set_bc": (C.c_int, [_vp, C.POINTER(C.c_int32)]),
    "ddg_curved_apply": (C.c_int, [_vp, C.c_int, C.c_double, _vp, _vp, _vp]),
    "ddg_curved_apply_dir": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp, _vp]),
    "ddg_curved_mass": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp]),
    "ddg_curved_rhs": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp, _vp, _vp]),
    "ddg_curved_pc_build": (C.c_int, [_vp, C.c_int, C.c_double, _vp]),
    "ddg_curved_pc_apply": (C.c_int, [_vp, _vp, _vp, _vp]),
    "ddg_curved_pc_blocks": (C.c_int, [_vp, _vp, _vp]),
    "ddg_curved_cg": (C.c_int, [_vp, C.c_int, C.POINTER(CgConfig), _vp, _vp, _vp, C.POINTER(SolveInfo)]),
    "ddg_sipg_set_kappa": (C.c_int, [_vp, _vp]),
    "ddg_sipg_grad_kappa": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "ddg_axpby": (C.c_int, [_i64, C.c_double, _vp, C.c_double, _vp, _vp]),
    "ddg_dot": (C.c_int, [_i64, C.c_int, _vp, _vp, _vp, _vp]),
    "ddg_cast": (C.c_int, [_i64, C.c_int, _vp, _vp, _vp]),
    "ddg_mesh_connect": (C.c_int, [_i64, _vp, _vp, _vp]),
    "ddg_mesh_maps": (C.c_int, [_i64, C.c_int32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                C.c_double, _vp, _vp]),
    "ddg_last_error": (C.c_char_p, []),
    "ddg_version": (C.c_char_p, []),
}

_lib = None


def lib():
    """Load (once) and return the shared library with typed prototypes."""
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            raise DdgError(-1, "load", f"{_LIB_PATH} is missing; run `python -m ddg_b200.build`")
        L = C.CDLL(_LIB_PATH)
        for name, (res, args) in _PROTOS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    return sorted(_PROTOS)


def check(code: int, where: str) -> None:
    if code != DDG_OK:
        raise DdgError(code, where, lib().ddg_last_error().decode())


def ptr(a) -> int:
    """Raw data pointer of a numpy array or torch tensor (None -> NULL)."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data


def stream_handle(stream=None) -> int:
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream
