"""ctypes binding of ``include/tdgl_b200.h`` (the in-tree ``libtdgl_b200.so``).

The library is built by ``nanowire_tdgl_b200/build.py``.  Loading fails with
an ImportError that says how to build it; there is no other implementation
to fall back to.
"""

from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtdgl_b200.so")

TDGL_OK, TDGL_ENOCONV, TDGL_EDTMIN, TDGL_EKMAX, TDGL_ENONFINITE, TDGL_ETIMEOUT, TDGL_EINVAL, TDGL_ECUDA, \
    TDGL_ENOMEM = range(9)
TDGL_FP64, TDGL_MIXED = 0, 1
TDGL_JVP_FD, TDGL_JVP_ANALYTIC, TDGL_JVP_KRYLOV = 0, 1, 2
TDGL_KRYLOV_GMRES, TDGL_KRYLOV_GCR = 0, 1


class GridDesc(C.Structure):
    _fields_ = [("Nx", C.c_int32), ("Ny", C.c_int32), ("Nz", C.c_int32),
                ("periodic_x", C.c_int32), ("periodic_y", C.c_int32), ("periodic_z", C.c_int32),
                ("hx", C.c_double), ("hy", C.c_double), ("hz", C.c_double), ("kappa", C.c_double)]


class MaterialDesc(C.Structure):
    _fields_ = [("hole_links", C.POINTER(C.c_int64) * 3), ("n_hole_links", C.c_int64 * 3),
                ("hole_interior", C.POINTER(C.c_int64) * 3), ("n_hole_interior", C.c_int64 * 3),
                ("kappa_full", C.POINTER(C.c_double)), ("sc_interior", C.POINTER(C.c_double))]


class Field(C.Structure):
    _fields_ = [("Bx", C.c_double), ("By", C.c_double), ("Bz", C.c_double),
                ("t_on_fraction", C.c_double), ("ramp_fraction", C.c_double), ("t_field_stop", C.c_double),
                ("ramp", C.c_int32), ("constant", C.c_int32)]


class TrapOpts(C.Structure):
    _fields_ = [("t_stop", C.c_double), ("dt", C.c_double), ("dt_min", C.c_double),
                ("newton_tol_f", C.c_double), ("newton_tol_dx", C.c_double), ("tol_gcr", C.c_double),
                ("eps_mf", C.c_double), ("newton_max_iter", C.c_int32), ("krylov_max_iter", C.c_int32),
                ("adaptive", C.c_int32), ("jvp_mode", C.c_int32)]


class Stats(C.Structure):
    _fields_ = [("status", C.c_int32), ("steps", C.c_int32), ("newton_converged", C.c_int32),
                ("newton_iters_last", C.c_int32), ("krylov_last", C.c_int32), ("max_krylov", C.c_int32),
                ("newton_iters", C.c_int64), ("krylov_iters", C.c_int64), ("rhs_evals", C.c_int64),
                ("jvp_evals", C.c_int64), ("rejections", C.c_int64), ("krylov_sq", C.c_int64), ("t", C.c_double), ("dt_cur", C.c_double),
                ("last_gnorm", C.c_double), ("last_dxnorm", C.c_double), ("kernel_launches", C.c_int64)]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


_P = C.c_void_p
_D = C.c_double
_I = C.c_int32

# name -> (restype, argtypes)
SIGNATURES = {
    "tdgl_ctx_create": (C.c_int, [C.POINTER(GridDesc), C.POINTER(MaterialDesc), _I, _I, C.POINTER(_P)]),
    "tdgl_ctx_destroy": (C.c_int, [_P]),
    "tdgl_ctx_set_krylov": (C.c_int, [_P, _I]),
    "tdgl_n_interior": (C.c_int64, [_P]),
    "tdgl_npad": (C.c_int64, [_P]),
    "tdgl_state_len": (C.c_int64, [_P]),
    "tdgl_workspace_bytes": (C.c_int64, [_P]),
    "tdgl_status_string": (C.c_char_p, [C.c_int]),
    "tdgl_last_error": (C.c_char_p, []),
    "tdgl_pack": (C.c_int, [_P, _P, _P, _P]),
    "tdgl_unpack": (C.c_int, [_P, _P, _P, _P]),
    "tdgl_rhs": (C.c_int, [_P, _P, _P, _D, _D, _D, _P]),
    "tdgl_eval_f": (C.c_int, [_P, _P, _P, _D, _D, _D, _P]),
    "tdgl_jvp": (C.c_int, [_P, _P, _P, _P, _D, _I, _D, _D, _D, _D, _P]),
    "tdgl_observables": (C.c_int, [_P, _P, _D, _D, _D, _P, _P, _P, _P, _P, _P, _P, _P]),
    "tdgl_tgcr_trap": (C.c_int, [_P, _P, _P, _P, _D, _D, _I, _D, _I, _D, _D, _D, C.POINTER(Stats), _P]),
    "tdgl_newton_trap": (C.c_int, [_P, _P, _P, _D, _D, _D, _I, _D, _D, _I, _D, _D, _D, C.POINTER(Stats), _P]),
    "tdgl_trap_run": (C.c_int, [_P, _P, C.POINTER(_D), C.POINTER(_D), _I, C.POINTER(TrapOpts), C.POINTER(Field),
                                C.POINTER(Stats), _P]),
    "tdgl_plaquette_winding": (C.c_int, [_P, _P, _D, _P, _P]),
    "tdgl_convergence_means": (C.c_int, [_P, _P, _P, _P, _P]),
    "tdgl_adjoint_solve": (C.c_int, [_P, _P, _P, _P, _D, _D, _D, _D, _D, C.POINTER(_I), _P]),
    "tdgl_trap_launch": (C.c_int, [_P, _P, _D, _D, _I, C.POINTER(TrapOpts), C.POINTER(Field), _P]),
    "tdgl_trap_collect": (C.c_int, [_P, C.POINTER(_D), C.POINTER(_D), C.POINTER(Stats)]),
    "tdgl_ctx_set_blocks": (C.c_int, [_P, _I, _I, _I]),
    "tdgl_ctx_set_poly": (C.c_int, [_P, _I]),
    "tdgl_ctx_set_limits": (C.c_int, [_P, C.c_int64, C.c_int64]),
    "tdgl_trap_launch_next": (C.c_int, [_P, _P, _I, C.POINTER(TrapOpts), C.POINTER(Field), _P]),
    "tdgl_ctx_poly_degree": (C.c_int32, [_P]),
    "tdgl_euler_run": (C.c_int, [_P, _P, C.POINTER(_D), _D, _D, _I, C.POINTER(Field), _P]),
    "tdgl_vjp": (C.c_int, [_P, _P, _P, _D, _D, _D, _P, _P, _P, _P, _P]),
    "tdgl_profile": (C.c_int, [_P, C.POINTER(C.c_uint64), C.c_int64, _I]),
    "tdgl_arnoldi_probe": (C.c_int, [_P, _I, _I, _I, _P]),
    "tdgl_eval_f_noalloc": (C.c_int, [C.POINTER(GridDesc), C.POINTER(MaterialDesc), _P, _P, _D, _D, _D, _P]),
}

_lib = None


def load() -> C.CDLL:
    """Load the shared library once; raise ImportError when it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m nanowire_tdgl_b200.build` "
            "(nvcc, sm_100a). The package has no CPU implementation.")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class TDGLError(RuntimeError):
    """A C-ABI call failed; ``status`` holds the tdgl_status code."""

    def __init__(self, status: int, where: str):
        lib = load()
        msg = lib.tdgl_status_string(status).decode()
        detail = lib.tdgl_last_error().decode()
        super().__init__(f"{where}: {msg}" + (f" ({detail})" if detail else ""))
        self.status = status


def check(status: int, where: str) -> int:
    if status != TDGL_OK:
        raise TDGLError(status, where)
    return status
