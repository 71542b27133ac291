"""ctypes binding of ``libsun_b200.so`` (the C ABI in ``include/sun_b200.h``).

The library is the product path; there is no fallback.  Loading fails loudly
when the shared object is missing -- build it with ``python -m sun_b200.build``.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsun_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "sun_b200.h")

STATUS = {0: "SUN_OK", 1: "SUN_ERR_INVALID_ARG", 2: "SUN_ERR_UNSUPPORTED", 3: "SUN_ERR_OUT_OF_MEMORY",
          4: "SUN_ERR_CUDA", 5: "SUN_ERR_IO", 6: "SUN_ERR_STATE", 7: "SUN_ERR_CAPACITY",
          8: "SUN_ERR_DEVICE_FLAG"}
SUN_OK = 0

SOA, SOA12, SOA8 = 0, 1, 2
EVEN_ODD, NORMAL = 0, 1
F32, F64 = 0, 1
HOST_CANONICAL, HOST_IMAGE = 0, 1


class SunConfig(C.Structure):
    _fields_ = [("device", C.c_int), ("verbosity", C.c_int), ("tune", C.c_int),
                ("tune_cache_path", C.c_char_p), ("hbm_budget_bytes", C.c_size_t)]


class SunLatticeParams(C.Structure):
    _fields_ = [("ncolors", C.c_int), ("dims", C.c_int * 4), ("beta", C.c_double), ("layout", C.c_int),
                ("order", C.c_int), ("precision", C.c_int), ("seed", C.c_uint64), ("reunit_every", C.c_int)]


class SunJob(C.Structure):
    _fields_ = [("ncolors", C.c_int), ("dims", C.c_int * 4), ("beta", C.c_double), ("sweeps", C.c_int),
                ("n_hb", C.c_int), ("n_or", C.c_int), ("seed", C.c_uint64), ("hot_start", C.c_int),
                ("observables", C.c_int), ("wilson_R", C.c_int), ("wilson_T", C.c_int),
                ("precision", C.c_int), ("layout", C.c_int), ("reunit_every", C.c_int)]


class SunServerStats(C.Structure):
    _fields_ = [("steps", C.c_int64), ("sweeps", C.c_int64), ("sweep_gpu_s", C.c_double), ("enqueue_s", C.c_double),
                ("admit_s", C.c_double), ("wait_s", C.c_double), ("retire_s", C.c_double), ("join_s", C.c_double)]


class SunResult(C.Structure):
    _fields_ = [("id", C.c_int64), ("status", C.c_int), ("plaquette", C.c_double * 2),
                ("polyakov", C.c_double * 2), ("wilson", C.c_double * (2 * 9 * 9)),
                ("submit_s", C.c_double), ("start_s", C.c_double), ("finish_s", C.c_double),
                ("link_updates", C.c_double)]


_vp = C.c_void_p
_dp = C.POINTER(C.c_double)
_SIGS = {
    "sun_init": [C.POINTER(SunConfig), C.POINTER(_vp)],
    "sun_finalize": [_vp],
    "sun_last_error_string": [_vp],
    "sun_version": [],
    "sun_lattice_create": [_vp, C.POINTER(SunLatticeParams), C.POINTER(_vp)],
    "sun_lattice_destroy": [_vp],
    "sun_lattice_bytes": [_vp, C.POINTER(C.c_size_t)],
    "sun_lattice_device_ptr": [_vp, C.POINTER(_vp)],
    "sun_lattice_init_cold": [_vp, _vp],
    "sun_lattice_init_hot": [_vp, _vp],
    "sun_lattice_upload": [_vp, _vp, C.c_int, _vp],
    "sun_lattice_download": [_vp, _vp, C.c_int, _vp],
    "sun_lattice_copy": [_vp, _vp, _vp],
    "sun_lattice_upload_async": [_vp, _vp, _vp],
    "sun_lattice_download_async": [_vp, _vp, _vp],
    "sun_lattice_get_rng": [_vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)],
    "sun_lattice_set_rng": [_vp, C.c_uint64, C.c_uint32, C.c_uint32],
    "sun_lattice_set_sweep_limit": [_vp, C.c_uint32],
    "sun_ctx_hbm_budget": [_vp, C.POINTER(C.c_size_t)],
    "sun_heatbath": [_vp, C.c_int, _vp],
    "sun_overrelax": [_vp, C.c_int, _vp],
    "sun_sweep": [_vp, C.c_int, C.c_int, C.c_int, _vp],
    "sun_sweep_measure": [_vp, C.c_int, C.c_int, C.c_int, _dp, _dp, _vp],
    "sun_heatbath_injected": [_vp, _vp, C.c_int, _vp],
    "sun_reunitarize": [_vp, _vp],
    "sun_unitarity_violation": [_vp, _dp, _vp],
    "sun_link_trace_det": [_vp, _dp, _vp],
    "sun_debug_fail_allocations": [C.c_int],
    "sun_debug_resident_barrier": [C.c_void_p, C.c_longlong, C.c_int],
    "sun_debug_su2_draws": [C.c_int, C.c_double, C.c_uint64, C.c_int, _dp],
    "sun_plaquette": [_vp, _dp, _vp],
    "sun_plaquette_noalloc": [_vp, C.POINTER(SunLatticeParams), _vp, _vp],
    "sun_polyakov": [_vp, _dp, _vp],
    "sun_wilson_loops": [_vp, C.c_int, C.c_int, _dp, _vp],
    "sun_smear_ape": [_vp, C.c_double, C.c_int, C.c_int, C.c_double, C.c_int, _vp],
    "sun_smear_stout": [_vp, C.c_double, C.c_int, C.c_int, _vp],
    "sun_smear_hyp": [_vp, _dp, C.c_int, C.c_int, C.c_double, C.c_int, _vp],
    "sun_multihit": [_vp, _vp, C.c_int, C.c_uint64, _vp],
    "sun_multihit_space": [_vp, _vp, C.c_int, _vp],
    "sun_save_bin": [_vp, C.c_char_p, C.c_int, C.c_int],
    "sun_load_bin": [_vp, C.c_char_p, C.c_int, C.c_int],
    "sun_batch_create": [_vp, C.POINTER(_vp)],
    "sun_batch_destroy": [_vp],
    "sun_batch_add": [_vp, _vp],
    "sun_batch_remove": [_vp, _vp],
    "sun_batch_size": [_vp, C.POINTER(C.c_int)],
    "sun_batch_sweep": [_vp, C.c_int, C.c_int, C.c_int, C.c_int, _vp],
    "sun_batch_plaquette": [_vp, _dp, _vp],
    "sun_batch_polyakov": [_vp, _dp, _vp],
    "sun_batch_wilson_loops": [_vp, C.c_int, C.c_int, _dp, _vp],
    "sun_server_create": [_vp, C.c_int, C.POINTER(_vp)],
    "sun_server_destroy": [_vp],
    "sun_server_submit": [_vp, C.POINTER(SunJob), C.POINTER(C.c_int64)],
    "sun_server_step": [_vp, C.POINTER(SunResult), C.c_int, C.POINTER(C.c_int)],
    "sun_server_pending": [_vp, C.POINTER(C.c_int), C.POINTER(C.c_int)],
    "sun_server_get_stats": [_vp, C.POINTER(SunServerStats)],
    "sun_job_footprint": [C.POINTER(SunJob), C.POINTER(C.c_size_t)],
    "sun_server_set_budget": [_vp, C.c_size_t],
    "sun_admit_count": [C.POINTER(C.c_size_t), C.c_int, C.c_size_t, C.c_size_t, C.c_int, C.POINTER(C.c_int)],
}

_lib = None


class SunError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


def lib() -> C.CDLL:
    """The loaded engine library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing; build it with `python -m sun_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        L.sun_last_error_string.restype = C.c_char_p
        L.sun_version.restype = C.c_char_p
        _lib = L
    return _lib


def check(status: int, ctx=None) -> None:
    if status != SUN_OK:
        msg = lib().sun_last_error_string(ctx)
        raise SunError(status, msg.decode() if msg else "")


def header_functions(path: str = HEADER):
    """Function names declared in the C header (for export checks)."""
    import re
    txt = open(path).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(sun_[a-z_0-9]+)\s*\(", txt)))
