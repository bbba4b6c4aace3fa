"""ctypes binding of libb200ldl.so (the C ABI in include/b200ldl.h).

The library is built in-tree by ``python -m amigo_b200.build``. There is no
fallback: if the library is missing or fails to load, every entry point
raises :class:`NativeError`.
"""

from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libb200ldl.so")

_i32p = ctypes.POINTER(ctypes.c_int)
_f64p = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p

# name -> (restype, argtypes); exactly the symbols declared in include/b200ldl.h
SIGNATURES = {
    "b200ldl_create": (ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int, ctypes.c_int, _i32p,
                                      _i32p, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_int]),
    "b200ldl_destroy": (None, [_vp]),
    "b200ldl_set_stream": (ctypes.c_int, [_vp, _vp]),
    "b200ldl_factor": (ctypes.c_int, [_vp, _vp, _vp]),
    "b200ldl_factor_host": (ctypes.c_int, [_vp, _f64p, _f64p]),
    "b200ldl_factor_elements": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    "b200ldl_solve": (ctypes.c_int, [_vp, ctypes.c_int, _vp, ctypes.c_int]),
    "b200ldl_solve_host": (ctypes.c_int, [_vp, ctypes.c_int, _f64p, ctypes.c_int]),
    "b200ldl_solve_refine": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, _vp, ctypes.c_int, _vp,
                                            ctypes.c_int, ctypes.c_int, ctypes.c_double, _f64p,
                                            _i32p]),
    "b200ldl_get_inertia": (ctypes.c_int, [_vp, _i32p, _i32p]),
    "b200ldl_set_precision": (ctypes.c_int, [_vp, ctypes.c_int]),
    "b200ldl_set_refinement": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double]),
    "b200ldl_last_refinement": (ctypes.c_int, [_vp, _i32p, _f64p, _i32p, _i32p]),
    "b200ldl_last_error": (ctypes.c_char_p, [_vp]),
    "b200ldl_symbolic_sizes": (ctypes.c_int, [_vp, _i32p, _i32p]),
    "b200ldl_get_symbolic": (ctypes.c_int, [_vp] + [_i32p] * 7),
    "b200ldl_node_pivots": (ctypes.c_int, [_vp, _i32p, _i32p]),
    "b200ldl_get_pivot_record": (ctypes.c_int, [_vp, _i32p, _i32p, _i32p, _i32p,
                                                ctypes.POINTER(ctypes.c_longlong)]),
    "b200ldl_set_pivot_record": (ctypes.c_int, [_vp, _i32p, _i32p, _i32p, _i32p]),
    "b200ldl_reuse_pivot_order": (ctypes.c_int, [_vp]),
    "b200ldl_stats": (ctypes.c_int, [_vp, _f64p, ctypes.c_int]),
    "b200ldl_set_profiling": (ctypes.c_int, [_vp, ctypes.c_int]),
    "b200ldl_reset_profile": (ctypes.c_int, [_vp]),
    "b200ldl_profile": (ctypes.c_int, [_vp, _f64p, ctypes.c_int]),
    "b200ldl_launch_count": (ctypes.c_longlong, [_vp]),
    "b200ldl_work": (ctypes.c_int, [_vp, _f64p, ctypes.c_int]),
    "b200ldl_schur_update_tc": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp,
                                               ctypes.c_int, _vp, ctypes.c_int, _vp,
                                               ctypes.c_int, ctypes.c_int, _vp]),
    "b200ldl_dense_solve_noalloc": (ctypes.c_int, [ctypes.c_int, _vp, ctypes.c_int, _vp,
                                                   ctypes.c_int, ctypes.c_int, _vp, _vp]),
    "b200ldl_create_batch": (ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int, _i32p, _i32p,
                                            _i32p, _i32p, ctypes.c_int, ctypes.c_double,
                                            ctypes.c_double, ctypes.c_double, ctypes.c_int]),
    "b200ldl_num_systems": (ctypes.c_int, [_vp]),
    "b200ldl_system_inertia": (ctypes.c_int, [_vp, _i32p, _i32p]),
    "b200ldl_value_gradient": (ctypes.c_int, [_vp, ctypes.c_int, _vp, ctypes.c_int, _vp,
                                              ctypes.c_int, _vp, _vp]),
    "b200ldl_set_perturbation_rows": (ctypes.c_int, [_vp, ctypes.c_int, _i32p, ctypes.c_int,
                                                     _i32p]),
    "b200ldl_factor_perturbed": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_double,
                                                ctypes.c_double, _i32p, _i32p]),
    "b200ldl_copy_perturbed_diagonal": (ctypes.c_int, [_vp, _vp]),
    "b200ldl_assembly_create": (ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int, _i32p, _i32p,
                                               ctypes.c_int, _i32p, _i32p, _i32p]),
    "b200ldl_assembly_values": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    "b200ldl_assembly_info": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_longlong),
                                             ctypes.c_int]),
    "b200ldl_assembly_plan": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_longlong),
                                             ctypes.POINTER(ctypes.c_longlong)]),
    "b200ldl_assembly_last_error": (ctypes.c_char_p, [_vp]),
    "b200ldl_assembly_destroy": (None, [_vp]),
}


class NativeError(RuntimeError):
    """A non-zero status from the native library (or the library is absent)."""

    def __init__(self, msg: str, status: int = -1):
        super().__init__(msg)
        self.status = status


_lib: ctypes.CDLL | None = None


def load() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise NativeError(
            f"{LIB_PATH} is missing; build it with `python -m amigo_b200.build`")
    try:
        lib = ctypes.CDLL(LIB_PATH)
    except OSError as e:  # pragma: no cover - depends on the machine
        raise NativeError(f"cannot load {LIB_PATH}: {e}") from e
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(handle, status: int, what: str) -> int:
    if status != 0:
        msg = load().b200ldl_last_error(handle)
        text = msg.decode() if msg else ""
        raise NativeError(f"{what} failed with status {status}: {text}", status)
    return status
