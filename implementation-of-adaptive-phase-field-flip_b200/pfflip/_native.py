"""ctypes binding of libpfflip.so, the sm_100a C ABI declared in include/pfflip.h.

There is no fallback: if the library is missing or cannot be loaded, every
entry point raises ``NativeError``.  Device buffers are torch CUDA tensors;
their raw pointers and the current torch stream cross the ABI as plain
integers.
"""

from __future__ import annotations

import ctypes as C
import os

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpfflip.so")

PF_OK = 0
PF_ERR_ARG = 1
PF_ERR_CUDA = 2
PF_ERR_NONFINITE = 3
PF_ERR_NOT_CONVERGED = 4
PF_ERR_WORKSPACE = 5
PF_ERR_UNSUPPORTED = 6

PF_SORT_STATIC_MAX_CELLS = 512 ** 3
PF_MG_MAX_LEVELS = 16
PF_MG_STATE_BYTES = 512
PF_MG_COUNTERS = 32
PF_PREC = {"fp32": 0, "fp16": 1, "bf16": 2}
PF_STENCIL = {"reference": 0, "flux": 1}


class NativeError(RuntimeError):
    """A libpfflip call failed (or the library is unavailable)."""

    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


class pf_grid(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("dx", C.c_float)]


class pf_mg_level(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("bx", C.c_void_p), ("by", C.c_void_p), ("bz", C.c_void_p), ("diag", C.c_void_p),
        ("p", C.c_void_p), ("p_alt", C.c_void_p), ("b", C.c_void_p), ("r", C.c_void_p),
        ("bx_lp", C.c_void_p), ("by_lp", C.c_void_p), ("bz_lp", C.c_void_p),
        ("p_lp", C.c_void_p), ("p_lp_alt", C.c_void_p), ("b_lp", C.c_void_p),
        ("bz_pad", C.c_void_p), ("bz_pitch", C.c_int32),
    ]


class pf_mg_desc(C.Structure):
    _fields_ = [
        ("nlev", C.c_int32),
        ("lev", pf_mg_level * PF_MG_MAX_LEVELS),
        ("omega", C.c_float),
        ("pre", C.c_int32), ("post", C.c_int32), ("coarsest", C.c_int32),
        ("precision", C.c_int32),
        ("stencil", C.c_int32),
        ("coef_scale", C.c_float),
        ("rhs", C.c_void_p), ("res_v", C.c_void_p), ("res_alt", C.c_void_p), ("z", C.c_void_p),
        ("q", C.c_void_p), ("Ap", C.c_void_p), ("x", C.c_void_p),
        ("state", C.c_void_p), ("partials", C.c_void_p), ("counters", C.c_void_p),
        ("bottom_op", C.c_void_p),
    ]


_lib = None
_VP, _I32, _I64, _F, _D = C.c_void_p, C.c_int32, C.c_int64, C.c_float, C.c_double
_G = C.POINTER(pf_grid)

# name -> (restype, argtypes); the list mirrors include/pfflip.h
SIGNATURES = {
    "pf_version": (C.c_char_p, []),
    "pf_last_error": (C.c_char_p, []),
    "pf_last_cuda_error": (C.c_int, []),
    "pf_launch_count": (C.c_uint64, []),
    "pf_sort_workspace_bytes": (C.c_size_t, [_G, _I64]),
    "pf_sort_particles": (C.c_int, [_G, _I64, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, C.c_size_t, _VP]),
    "pf_sort_particles_static": (C.c_int, [_G, _I64] + [_VP] * 7 + [_VP]),
    "pf_p2g": (C.c_int, [_G, _I64, _VP, _VP, _VP, _F, _F, _F] + [_VP] * 8 + [_VP]),
    "pf_phase_beta": (C.c_int, [_G] + [_VP] * 7 + [_VP] + [_F] * 6 + [_VP] * 14 + [_VP]),
    "pf_save_and_force": (C.c_int, [_G] + [_VP] * 6 + [_VP, _F, _F, _F, _F, _VP]),
    "pf_build_rhs": (C.c_int, [_G, _VP, _VP, _VP, _VP, _VP, _F, _F, _F, _VP]),
    "pf_project": (C.c_int, [_G, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _F, _VP]),
    "pf_max_divergence": (C.c_int, [_G, _VP, _VP, _VP, _VP, _VP]),
    "pf_extrapolate": (C.c_int, [_G, _VP, _VP, _VP, _VP, _I32, _VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    "pf_g2p_advect": (C.c_int, [_G, _I64, _VP, _VP] + [_VP] * 9 + [_VP, _F, _F, _F, C.POINTER(_F),
                                                                     C.POINTER(_F), _I32, _I32, _VP]),
    "pf_g2p_workspace_bytes": (C.c_size_t, [_G]),
    "pf_g2p_advect_packed": (C.c_int, [_G, _I64, _VP, _VP] + [_VP] * 9 + [_VP, _F, _F, _F, C.POINTER(_F),
                                                                          C.POINTER(_F), _I32, _I32, _VP, _VP,
                                                                          C.c_size_t, _VP]),
    "pf_particle_max_speed": (C.c_int, [_I64, _VP, _VP, _VP, _VP]),
    "pf_droplet_classify": (C.c_int, [_G, _I64, _VP, _VP, _VP, _VP, _F, _F, _F, _F, _F, C.c_uint32, _VP, _VP]),
    "pf_velocity_gradient": (C.c_int, [_G, _VP, _VP, _VP, _VP, _VP]),
    "pf_spray_emit": (C.c_int, [_G, _I64, _VP, _VP, _VP, _VP, _VP, _F, _F, _F, _F, _F, _F, C.c_uint32, _VP, _VP]),
    "pf_droplet_advance": (C.c_int, [_G, _I64, _VP, _VP, _VP, _VP, _VP, _VP, _F, C.POINTER(_F), _F, _F, _F, _F, _F,
                                     C.POINTER(_F), C.POINTER(_F), _I32, _VP]),
    "pf_spray_rasterize": (C.c_int, [_I64, _VP, _VP, _VP, _I32, _I32, _I32, _F, _VP]),
    "pf_permute_f32": (C.c_int, [_I64, _VP, _VP, _VP, _VP]),
    "pf_apply_A": (C.c_int, [_G, _VP, _VP, _VP, _VP, _VP, _VP, _I32, _VP]),
    "pf_mg_partials_count": (C.c_int64, []),
    "pf_mg_level_count": (C.c_int32, [_I32, _I32, _I32, _I32, C.POINTER(_I32)]),
    "pf_mg_plan_create": (C.c_int, [C.POINTER(pf_mg_desc), C.POINTER(_VP)]),
    "pf_mg_plan_destroy": (C.c_int, [_VP]),
    "pf_mg_bottom_info": (C.c_int, [_VP, C.POINTER(_I32), C.POINTER(_I32), C.POINTER(_I32)]),
    "pf_mg_bottom_op_floats": (C.c_int64, [C.POINTER(pf_mg_desc)]),
    "pf_mg_build_hierarchy": (C.c_int, [_VP, _VP, _VP, _VP, _VP]),
    "pf_mg_precondition": (C.c_int, [_VP, _VP, _VP, _VP]),
    "pf_mg_smooth": (C.c_int, [_VP, _I32, _I32, _I32, _VP]),
    "pf_mg_solve": (C.c_int, [_VP, _VP, _VP, _F, _I32, _I32, _I32, C.POINTER(_I32), C.POINTER(_D), _VP]),
    "pf_adj_g2p_advect": (C.c_int, [_G, _I64, _VP, _VP] + [_VP] * 9 + [_F, _F, _F, C.POINTER(_F), C.POINTER(_F),
                                                                       _I32, _I32] + [_VP] * 4 + [_VP] * 9 + [_VP]),
    "pf_adj_extrapolate": (C.c_int, [_G, _VP, _I32] + [_VP] * 15 + [_VP]),
    "pf_adj_project": (C.c_int, [_G] + [_VP] * 7 + [_F] + [_VP] * 4 + [_VP]),
    "pf_adj_face_sources": (C.c_int, [_G] + [_VP] * 11 + [_VP] + [_F] * 7 + [_VP] * 15 + [_VP]),
    "pf_adj_p2g": (C.c_int, [_G, _I64, _VP, _VP, _F, _F, _F] + [_VP] * 7 + [_VP, _VP, _VP]),
    "pf_adj_phase_cell": (C.c_int, [_G, _VP, _VP, _F, _F, _F, _VP, _VP]),
    "pf_adj_unsort": (C.c_int, [_I64, _VP, _VP, _VP, _VP, _VP, _VP]),
}


def lib():
    """The loaded library (raises NativeError when it is not available)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise NativeError(-1, f"libpfflip.so not built ({LIB_PATH}); run build.py")
        try:
            L = C.CDLL(LIB_PATH)
        except OSError as e:  # pragma: no cover
            raise NativeError(-1, f"cannot load {LIB_PATH}: {e}") from e
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name, None)
            if f is None:
                continue
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    return lib().pf_last_error().decode(errors="replace")


def check(rc: int, what: str, ok=(PF_OK,)):
    if rc not in ok:
        raise NativeError(rc, f"{what} failed: {last_error()}")
    return rc


def call(name: str, *args, ok=(PF_OK,)):
    return check(getattr(lib(), name)(*args), name, ok=ok)


def sptr(t) -> int:
    """Device address of a particle stream.  The simulator's streams are views
    of the first n rows of at least one row of storage, so an empty stream
    still has its storage's address (torch reports 0 for an empty tensor)."""
    return t.untyped_storage().data_ptr() + t.storage_offset() * t.element_size()


def ptr(t) -> int | None:
    """Raw device pointer of a tensor (or of a DeviceArray), None for None."""
    if t is None:
        return None
    if hasattr(t, "tensor"):
        t = t.tensor
    return t.data_ptr()


def stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def grid(res, dx) -> pf_grid:
    return pf_grid(int(res[0]), int(res[1]), int(res[2]), float(dx))


def require_cuda(device) -> torch.device:
    dev = torch.device(device)
    if dev.type != "cuda":
        raise NativeError(PF_ERR_UNSUPPORTED, f"device {device!r}: this implementation runs on CUDA devices only")
    if not torch.cuda.is_available():
        raise NativeError(PF_ERR_CUDA, "no CUDA device is available")
    lib()
    return dev


def launch_count() -> int:
    return int(lib().pf_launch_count())
