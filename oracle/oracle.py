"""ctypes front-end of the FP64 CPU oracle (``oracle/libsun_oracle.so``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py``'s CPU-baseline leg as the checker.  The product never imports
this module.

Lattices are numpy ``complex128`` arrays of shape ``(V, 4, N, N)`` in the
canonical order (lexicographic sites, x fastest), the record order of the
reference's ``SaveBin_Gauge`` file body (src/io_gauge.cpp:544-563).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libsun_oracle.so")

RNG_PHILOX32 = 0
RNG_PHILOX64 = 1
RNG_INJECTED = 2
SOA, SOA12, SOA8 = 0, 1, 2

_lib = None


def build() -> None:
    """Compile the oracle (gcc, OpenMP) in place."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_u32p = C.POINTER(C.c_uint32)


def _declare(L: C.CDLL) -> None:
    L.orc_philox4x32_10.argtypes = [_u32p, _u32p, _u32p]
    L.orc_uniforms.argtypes = [C.c_uint64, C.c_int, C.c_int, C.c_int, C.c_uint32, C.c_int, C.c_int, _dp]
    L.orc_su2_index.argtypes = [C.c_int, C.c_int, _ip, _ip]
    L.orc_reunit_link.argtypes = [C.c_int, _dp]
    L.orc_heatbath_link.argtypes = [C.c_int, _dp, _dp, C.c_double, C.c_int, C.c_uint64, C.c_int,
                                    C.c_int, C.c_uint32, _dp, C.c_int]
    L.orc_heatbath_link.restype = C.c_int
    L.orc_overrelax_link.argtypes = [C.c_int, _dp, _dp]
    L.orc_su2_generate.argtypes = [C.c_double, C.c_int, C.c_uint64, C.c_int, C.c_int, C.c_uint32,
                                   _dp, C.c_int, _dp, _ip]
    L.orc_cold.argtypes = [C.c_int, _ip, _dp]
    L.orc_hot.argtypes = [C.c_int, _ip, _dp, C.c_uint64]
    L.orc_staple.argtypes = [C.c_int, _ip, _dp, C.c_int, C.c_int, _dp]
    L.orc_update_phase.argtypes = [C.c_int, _ip, _dp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int,
                                   C.c_uint64, C.c_uint32, _dp, C.c_int, C.c_int]
    L.orc_update_phase.restype = C.c_int
    L.orc_sweeps.argtypes = [C.c_int, _ip, _dp, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int,
                             C.c_int, C.c_uint64, _u32p, C.c_int]
    L.orc_reunitarize.argtypes = [C.c_int, _ip, _dp]
    L.orc_unitarity_violation.argtypes = [C.c_int, _ip, _dp]
    L.orc_unitarity_violation.restype = C.c_double
    L.orc_link_trace_det.argtypes = [C.c_int, _ip, _dp, _dp]
    L.orc_plaquette.argtypes = [C.c_int, _ip, _dp, _dp]
    L.orc_polyakov.argtypes = [C.c_int, _ip, _dp, _dp]
    L.orc_wilson_loops.argtypes = [C.c_int, _ip, _dp, C.c_int, C.c_int, _dp]
    L.orc_layout_elems.argtypes = [C.c_int, C.c_int]
    L.orc_layout_elems.restype = C.c_int
    L.orc_pack.argtypes = [C.c_int, _ip, _dp, C.c_int, C.c_int, C.c_int, C.c_void_p]
    L.orc_unpack.argtypes = [C.c_int, _ip, C.c_void_p, C.c_int, C.c_int, C.c_int, _dp]
    L.orc_save_bin.argtypes = [C.c_int, _ip, _dp, C.c_double, C.c_char_p, C.c_int, C.c_int, C.c_int]
    L.orc_save_bin.restype = C.c_int
    L.orc_load_bin.argtypes = [C.c_int, _ip, _dp, C.c_char_p, C.c_int, C.c_int, C.c_int, _ip, _dp]
    L.orc_load_bin.restype = C.c_int
    L.orc_project_sun.argtypes = [C.c_int, _dp, _dp, C.c_int, C.c_double]
    L.orc_exp_iq3.argtypes = [_dp, _dp]
    L.orc_ape.argtypes = [C.c_int, _ip, _dp, C.c_double, C.c_int, C.c_int, C.c_double, C.c_int]
    L.orc_stout.argtypes = [_ip, _dp, C.c_double, C.c_int, C.c_int]
    L.orc_hyp.argtypes = [C.c_int, _ip, _dp, C.POINTER(C.c_float), C.c_int, C.c_int, C.c_double, C.c_int]
    L.orc_multihit.argtypes = [C.c_int, _ip, _dp, _dp, C.c_double, C.c_int, C.c_int, C.c_uint64]
    L.orc_multihit_space.argtypes = [C.c_int, _ip, _dp, _dp, C.c_int]


def _d(a: np.ndarray):
    assert a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def _dims(X):
    return (C.c_int * 4)(*[int(v) for v in X])


def volume(X) -> int:
    return int(X[0]) * int(X[1]) * int(X[2]) * int(X[3])


def empty(N: int, X) -> np.ndarray:
    return np.zeros((volume(X), 4, N, N), dtype=np.complex128)


def philox4x32_10(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().orc_philox4x32_10(c, k, o)
    return [int(v) for v in o]


def uniforms(seed, lex, mu, n, fp64=False, purpose=0, pass_=0):
    out = np.zeros(n)
    lib().orc_uniforms(seed, lex, mu, purpose, pass_, int(bool(fp64)), n, _d(out))
    return out


def su2_index(N: int, block: int):
    p, q = C.c_int(), C.c_int()
    lib().orc_su2_index(N, block, C.byref(p), C.byref(q))
    return p.value, q.value


def reunit_link(U: np.ndarray) -> np.ndarray:
    U = np.ascontiguousarray(U, dtype=np.complex128).copy()
    lib().orc_reunit_link(U.shape[0], _d(U))
    return U


def heatbath_link(U, F, beta_over_n, mode=RNG_PHILOX64, seed=0, lex=0, mu=0, pass_=0, inj=None):
    U = np.ascontiguousarray(U, dtype=np.complex128).copy()
    F = np.ascontiguousarray(F, dtype=np.complex128)
    injp = _d(inj) if inj is not None else None
    used = lib().orc_heatbath_link(U.shape[0], _d(U), _d(F), beta_over_n, mode, seed, lex, mu, pass_,
                                   injp, 0 if inj is None else len(inj))
    return U, used


def overrelax_link(U, F):
    U = np.ascontiguousarray(U, dtype=np.complex128).copy()
    F = np.ascontiguousarray(F, dtype=np.complex128)
    lib().orc_overrelax_link(U.shape[0], _d(U), _d(F))
    return U


def su2_generate(alpha, mode=RNG_PHILOX64, seed=0, lex=0, mu=0, pass_=0, inj=None):
    a = np.zeros(4)
    used = C.c_int()
    injp = _d(inj) if inj is not None else None
    lib().orc_su2_generate(alpha, mode, seed, lex, mu, pass_, injp, 0 if inj is None else len(inj),
                           _d(a), C.byref(used))
    return a, used.value


def cold(N, X):
    U = empty(N, X)
    lib().orc_cold(N, _dims(X), _d(U))
    return U


def hot(N, X, seed):
    U = empty(N, X)
    lib().orc_hot(N, _dims(X), _d(U), seed)
    return U


def staple(U, X, lex, mu):
    N = U.shape[-1]
    S = np.zeros((N, N), dtype=np.complex128)
    lib().orc_staple(N, _dims(X), _d(U), lex, mu, _d(S))
    return S


def update_phase(U, X, parity, mu, kind, beta, mode=RNG_PHILOX64, seed=0, pass_=0, inj=None,
                 inj_stride=0, nthreads=0):
    """In place.  kind 0 = heatbath, 1 = overrelaxation."""
    N = U.shape[-1]
    injp = _d(inj) if inj is not None else None
    return lib().orc_update_phase(N, _dims(X), _d(U), parity, mu, kind, beta, mode, seed, pass_,
                                  injp, inj_stride, nthreads)


def sweeps(U, X, beta, n_hb, n_or, n_sweeps, reunit_every=0, mode=RNG_PHILOX64, seed=0, pass_=0,
           nthreads=0):
    """In place; returns the heatbath-pass counter after the sweeps."""
    N = U.shape[-1]
    p = C.c_uint32(pass_)
    lib().orc_sweeps(N, _dims(X), _d(U), beta, n_hb, n_or, n_sweeps, reunit_every, mode, seed,
                     C.byref(p), nthreads)
    return p.value


def reunitarize(U, X):
    lib().orc_reunitarize(U.shape[-1], _dims(X), _d(U))


def unitarity_violation(U, X) -> float:
    return lib().orc_unitarity_violation(U.shape[-1], _dims(X), _d(U))


def link_trace_det(U, X):
    o = np.zeros(4)
    lib().orc_link_trace_det(U.shape[-1], _dims(X), _d(U), _d(o))
    return o


def plaquette(U, X):
    o = np.zeros(2)
    lib().orc_plaquette(U.shape[-1], _dims(X), _d(U), _d(o))
    return o


def polyakov(U, X):
    o = np.zeros(2)
    lib().orc_polyakov(U.shape[-1], _dims(X), _d(U), _d(o))
    return o


def wilson_loops(U, X, R, T):
    o = np.zeros(2 * (R + 1) * (T + 1))
    lib().orc_wilson_loops(U.shape[-1], _dims(X), _d(U), R, T, _d(o))
    return o.reshape(R + 1, T + 1, 2)


def layout_elems(N, layout):
    return lib().orc_layout_elems(N, layout)


def pack(U, X, layout=SOA, evenodd=True, fp64=True) -> np.ndarray:
    N = U.shape[-1]
    ne = layout_elems(N, layout)
    img = np.zeros(ne * 4 * volume(X), dtype=np.complex128 if fp64 else np.complex64)
    lib().orc_pack(N, _dims(X), _d(U), layout, int(evenodd), int(fp64), img.ctypes.data)
    return img


def unpack(img, N, X, layout=SOA, evenodd=True) -> np.ndarray:
    fp64 = img.dtype == np.complex128
    U = empty(N, X)
    img = np.ascontiguousarray(img)
    lib().orc_unpack(N, _dims(X), img.ctypes.data, layout, int(evenodd), int(fp64), _d(U))
    return U


def save_bin(U, X, beta, path, save_fp64=True, header_fp64=True, with_header=True):
    return lib().orc_save_bin(U.shape[-1], _dims(X), _d(U), beta, path.encode(), int(save_fp64),
                              int(header_fp64), int(with_header))


def load_bin(N, X, path, save_fp64=True, header_fp64=True, with_header=True):
    U = empty(N, X)
    g = (C.c_int * 4)()
    b = C.c_double()
    rc = lib().orc_load_bin(N, _dims(X), _d(U), path.encode(), int(save_fp64), int(header_fp64),
                            int(with_header), g, C.byref(b))
    return rc, U, list(g), b.value


# -- smearing and multihit (src/smear/*.cu); dirmask bit mu selects direction mu
SPACE, TIME = 7, 8


def project_sun(W, Q, nhits, tol=0.0):
    """Projection of Q onto SU(N) started from W (project_link / SU3project)."""
    W = np.ascontiguousarray(W, dtype=np.complex128).copy()
    Q = np.ascontiguousarray(Q, dtype=np.complex128)
    lib().orc_project_sun(W.shape[-1], _d(W), _d(Q), nhits, tol)
    return W


def exp_iq3(Q):
    Q = np.ascontiguousarray(Q, dtype=np.complex128)
    E = np.zeros((3, 3), dtype=np.complex128)
    lib().orc_exp_iq3(_d(Q), _d(E))
    return E


def ape(U, X, w, steps, nhits, tol, dirmask):
    """In place."""
    lib().orc_ape(U.shape[-1], _dims(X), _d(U), w, steps, nhits, tol, dirmask)


def stout(U, X, w, steps, dirmask):
    """In place (SU(3))."""
    assert U.shape[-1] == 3
    lib().orc_stout(_dims(X), _d(U), w, steps, dirmask)


def hyp(U, X, alpha, steps, nhits, tol, dirmask):
    """In place; alpha = (alpha1, alpha2, alpha3), stored as FP32."""
    a = (C.c_float * 3)(*[float(v) for v in alpha])
    lib().orc_hyp(U.shape[-1], _dims(X), _d(U), a, steps, nhits, tol, dirmask)


def multihit(U, X, beta, nhit, seed, mode=RNG_PHILOX64):
    out = np.empty_like(U)
    lib().orc_multihit(U.shape[-1], _dims(X), _d(U), _d(out), beta, nhit, mode, seed)
    return out


def multihit_space(U, X, nhit):
    out = np.empty_like(U)
    lib().orc_multihit_space(U.shape[-1], _dims(X), _d(U), _d(out), nhit)
    return out
