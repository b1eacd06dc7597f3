"""ctypes bindings of libimpeller_msm.so (the C ABI in include/impeller_msm.h).

There is no fallback: if the CUDA library is missing or fails to load, every
entry point raises.  The library is built in-tree by ``impeller_b200.build``.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libimpeller_msm.so")

c_u32p = ctypes.POINTER(ctypes.c_uint32)
c_u32pp = ctypes.POINTER(c_u32p)
c_void_pp = ctypes.POINTER(ctypes.c_void_p)
c_ulong_p = ctypes.POINTER(ctypes.c_ulong)


class PolyPtr(ctypes.Structure):
    """include/impeller_ntt.h PolyPtr (core/src/common/iter/src/iter.cuh:12-18)."""
    _fields_ = [("ptr", ctypes.c_void_p), ("len", ctypes.c_size_t), ("rotate", ctypes.c_size_t),
                ("offset", ctypes.c_size_t), ("whole_len", ctypes.c_size_t)]


class PolySlice(ctypes.Structure):
    """include/impeller_ntt.h PolySlice (core/src/common/slice/poly_slice.h:4-12)."""
    _fields_ = [("begin", ctypes.c_ulonglong), ("slice_len", ctypes.c_ulonglong), ("len", ctypes.c_ulonglong)]


_u32 = ctypes.c_uint
_cptr = ctypes.c_void_p

# Every symbol include/impeller_msm.h and include/impeller_ntt.h declare, with (restype, argtypes).
SIGNATURES: dict[str, tuple] = {
    "msm": (ctypes.c_int, [c_void_pp, c_ulong_p, ctypes.c_ulonglong, ctypes.c_uint, ctypes.c_uint, ctypes.c_uint,
                           ctypes.c_uint, ctypes.c_uint, c_u32p, c_u32pp, ctypes.c_uint, c_u32pp, c_u32pp]),
    "msm_precompute": (ctypes.c_int, [ctypes.c_ulonglong, c_u32pp, ctypes.c_uint]),
    "impeller_msm_cfg": (ctypes.c_int, [ctypes.c_uint, ctypes.c_uint, ctypes.c_int, c_void_pp, c_ulong_p,
                                        ctypes.c_ulonglong, ctypes.c_uint, ctypes.c_uint, ctypes.c_uint,
                                        ctypes.c_uint, ctypes.c_uint, c_u32p, c_u32pp, ctypes.c_uint, c_u32pp,
                                        c_u32pp]),
    "impeller_msm_precompute_cfg": (ctypes.c_int, [ctypes.c_uint, ctypes.c_uint, ctypes.c_ulonglong, c_u32pp,
                                                   ctypes.c_uint]),
    "impeller_msm_n_precompute": (ctypes.c_uint, [ctypes.c_uint, ctypes.c_uint]),
    "impeller_msm_cfg_curve": (ctypes.c_int, [ctypes.c_uint, ctypes.c_uint, ctypes.c_uint, ctypes.c_int, c_void_pp,
                                              c_ulong_p, ctypes.c_ulonglong, ctypes.c_uint, ctypes.c_uint,
                                              ctypes.c_uint, ctypes.c_uint, ctypes.c_uint, c_u32p, c_u32pp,
                                              ctypes.c_uint, c_u32pp, c_u32pp]),
    "impeller_msm_precompute_cfg_curve": (ctypes.c_int, [ctypes.c_uint, ctypes.c_uint, ctypes.c_uint,
                                                         ctypes.c_ulonglong, c_u32pp, ctypes.c_uint]),
    "impeller_msm_n_precompute_curve": (ctypes.c_uint, [ctypes.c_uint, ctypes.c_uint, ctypes.c_uint]),
    "impeller_ctx_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.c_void_p,
                                           ctypes.c_uint64, ctypes.c_int]),
    "impeller_ctx_create_curve": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.c_void_p,
                                                 ctypes.c_uint64, ctypes.c_int, ctypes.c_uint]),
    "impeller_ctx_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "impeller_ctx_points": (ctypes.c_void_p, [ctypes.c_void_p]),
    "impeller_ctx_len": (ctypes.c_uint64, [ctypes.c_void_p]),
    "impeller_ctx_precompute": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint]),
    "impeller_ctx_window": (ctypes.c_uint, [ctypes.c_void_p, ctypes.c_uint64]),
    "impeller_default_window": (ctypes.c_uint, [ctypes.c_uint64]),
    "impeller_default_window_curve": (ctypes.c_uint, [ctypes.c_uint64, ctypes.c_uint]),
    "impeller_table_window": (ctypes.c_uint, [ctypes.c_uint64]),
    "impeller_set_window_table": (ctypes.c_int, [c_u32p, c_u32p, c_u32p, ctypes.c_uint32]),
    "impeller_msm_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint,
                                           ctypes.c_void_p, ctypes.c_void_p]),
    "impeller_msm_host": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint,
                                         ctypes.c_void_p, ctypes.c_void_p]),
    "impeller_batch_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p,
                                             ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint),
                                             ctypes.c_uint32, ctypes.c_uint32]),
    "impeller_batch_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "impeller_batch_run": (ctypes.c_int, [ctypes.c_void_p, c_void_pp, ctypes.c_void_p, ctypes.c_void_p]),
    "impeller_batch_launches": (ctypes.c_uint32, [ctypes.c_void_p]),
    "impeller_batch_profile": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "impeller_batch_profile_read": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_uint32,
                                                   ctypes.POINTER(ctypes.c_uint32)]),
    "impeller_server_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p, ctypes.c_uint32,
                                              ctypes.c_uint32, ctypes.c_uint64]),
    "impeller_server_submit": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                              ctypes.POINTER(ctypes.c_uint64)]),
    "impeller_server_wait": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                                            ctypes.POINTER(ctypes.c_double)]),
    "impeller_server_poll": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                                            ctypes.POINTER(ctypes.c_double)]),
    "impeller_server_get_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "impeller_server_inject_failures": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32]),
    "impeller_server_fail_setup_step": (ctypes.c_int, [ctypes.c_uint32]),
    "impeller_server_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "impeller_gen_scalars": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64,
                                            ctypes.c_int, ctypes.c_uint64, ctypes.c_int, ctypes.c_void_p]),
    "impeller_gen_points": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64,
                                           ctypes.c_void_p]),
    "impeller_gen_scalars_curve": (ctypes.c_int, [ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64,
                                                  ctypes.c_uint64, ctypes.c_int, ctypes.c_uint64, ctypes.c_int,
                                                  ctypes.c_void_p]),
    "impeller_gen_points_curve": (ctypes.c_int, [ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64,
                                                 ctypes.c_uint64, ctypes.c_void_p]),
    "impeller_test_field_op": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                              ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]),
    "impeller_test_point_op": (ctypes.c_int, [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                              ctypes.c_uint64, ctypes.c_void_p]),
    "impeller_test_point_op_curve": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                                    ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]),
    "impeller_ctx_profile": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "impeller_ctx_profile_read": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_uint32,
                                                 ctypes.POINTER(ctypes.c_uint32)]),
    "impeller_phase_name": (ctypes.c_char_p, [ctypes.c_uint32]),
    "impeller_ctx_launches": (ctypes.c_uint32, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint]),
    "impeller_imad_peak": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
    "impeller_imad_peak_curve": (ctypes.c_int, [ctypes.c_int, ctypes.c_uint, ctypes.POINTER(ctypes.c_double)]),
    "impeller_op_latency": (ctypes.c_int, [ctypes.c_int, ctypes.c_uint32, ctypes.POINTER(ctypes.c_double)]),
    "impeller_msm_device_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                                                   ctypes.c_void_p]),
    "ssip_ntt": (ctypes.c_int, [PolyPtr, _cptr, _u32, _cptr, _u32, _u32]),
    "ssip_precompute": (ctypes.c_int, [_cptr, _u32, _cptr]),
    "recompute_ntt": (ctypes.c_int, [PolyPtr, _cptr, _u32, _cptr, _u32, _cptr, _u32, _u32]),
    "gen_pq_omegas": (None, [_cptr, _cptr, _u32, _u32, _cptr]),
    "distribute_powers": (ctypes.c_int, [PolyPtr, _cptr, ctypes.c_ulonglong, _cptr, ctypes.POINTER(PolySlice)]),
    "impeller_ntt": (ctypes.c_int, [ctypes.c_int, PolyPtr, _cptr, _u32, _cptr]),
    "impeller_ntt_precompute": (ctypes.c_int, [ctypes.c_int, _cptr, _u32, _cptr]),
    "impeller_ntt_recompute": (ctypes.c_int, [ctypes.c_int, PolyPtr, _cptr, _u32, _cptr]),
    "impeller_ntt_gen_pq_omegas": (ctypes.c_int, [ctypes.c_int, _cptr, _cptr, _u32, _u32, _cptr]),
    "impeller_ntt_distribute_powers": (ctypes.c_int, [ctypes.c_int, PolyPtr, _cptr, ctypes.c_ulonglong, _cptr,
                                                      ctypes.POINTER(PolySlice)]),
    "impeller_ntt_launches": (_u32, [_u32]),
    "impeller_last_error": (ctypes.c_char_p, []),
    "impeller_version": (ctypes.c_char_p, []),
}

_lib = None


class ImpellerError(RuntimeError):
    pass


def load(path: str | None = None):
    """Load the CUDA library (once).  Raises if it is not built."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise ImpellerError(f"{p} is missing: build it with `python -m impeller_b200.build` "
                            "(there is no CPU fallback)")
    L = ctypes.CDLL(p, mode=ctypes.RTLD_GLOBAL)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = L
    return L


def check(rc: int, what: str = "") -> None:
    if rc != 0:
        msg = load().impeller_last_error().decode(errors="replace")
        raise ImpellerError(f"{what or 'impeller call'} failed with cudaError {rc}: {msg}")


HEADERS = ("impeller_msm.h", "impeller_ntt.h")


def declared_symbols(header: str | None = None) -> list[str]:
    """Function names declared in include/impeller_msm.h and include/impeller_ntt.h
    (or in one given header), in declaration order."""
    import re
    inc = os.path.join(os.path.dirname(HERE), "include")
    keep = []
    for h in ([header] if header else [os.path.join(inc, name) for name in HEADERS]):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for n in re.findall(r"\b([A-Za-z_]\w*)\s*\(", text):
            if n in ("if", "sizeof", "defined") or n.isupper() or n in keep:
                continue
            keep.append(n)
    return keep
