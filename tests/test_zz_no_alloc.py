"""The allocation-free plaquette entry point, sun_plaquette_noalloc.

It exists for callers that cannot let a library call cudaMalloc:
applications whose device memory all belongs to their own pool, hosts with a
fixed memory budget, and loops that cannot afford the synchronisation of a
later cudaFree.  Its scratch is a fixed
array compiled into the library; these tests call it through the C ABI and
check it against the allocating sun_plaquette on two calls in a row.

The file name sorts last so that a run stopping at the first failure has run
every other test before this one.
"""
import ctypes as C

import pytest

pytestmark = pytest.mark.gpu

CASES = [(3, (8, 8, 8, 8), 1, "f32", True), (3, (4, 4, 4, 8), 0, "f64", True), (3, (4, 4, 4, 4), 2, "f64", True),
         (2, (4, 4, 4, 4), 0, "f32", True), (4, (4, 4, 6, 4), 0, "f64", True), (6, (4, 4, 4, 4), 0, "f32", True),
         (3, (4, 6, 4, 8), 1, "f32", False), (4, (4, 4, 4, 6), 0, "f64", False)]


def _params(N, dims, lay, prec, evenodd=True):
    from sun_b200._native import SunLatticeParams
    return SunLatticeParams(N, (C.c_int * 4)(*dims), 0.0, lay, 0 if evenodd else 1, 1 if prec == "f64" else 0, 0, 0)


@pytest.mark.parametrize("N,dims,lay,prec,evenodd", CASES)
def test_noalloc_plaquette_matches_allocating_entry_point(ctx, N, dims, lay, prec, evenodd):
    """Two calls in a row, on two configurations, against sun_plaquette (to
    1e-12) and against the oracle's plaquette of the same stored links; both
    storage orders.  Library allocations are switched off around the calls:
    one attempted through the library would fail them."""
    import torch
    from oracle import oracle as O
    from sun_b200 import HeatBath, PlaquetteCUB, gauge
    from sun_b200._native import lib
    g = gauge(ctx, N=N, dims=dims, beta={2: 2.3, 3: 5.9, 4: 10.5, 6: 25.0}[N], atype=lay, prec=prec, seed=3,
              evenodd=evenodd)
    g.Init(hot=True)
    p = _params(N, dims, lay, prec, evenodd)
    out = torch.full((2,), -1.0, dtype=torch.float64, device="cuda")
    for call in range(2):
        if call == 1:
            # a different configuration for the second call (updates need
            # even/odd arrays: a lexicographic lattice gets a new hot start)
            if evenodd:
                HeatBath(g).Run(1)
            else:
                g.Set(O.hot(N, list(dims), 11))
        torch.cuda.synchronize()
        assert lib().sun_debug_fail_allocations(0) == 0
        try:
            st = lib().sun_plaquette_noalloc(C.c_void_p(g.GetPtr()), C.byref(p), C.c_void_p(out.data_ptr()), None)
        finally:
            lib().sun_debug_fail_allocations(-1)
        assert st == 0, lib().sun_last_error_string(None)
        torch.cuda.synchronize()
        got = out.cpu().tolist()
        ref = PlaquetteCUB(g).Run()
        assert abs(got[0] - ref.real) < 1e-12 and abs(got[1] - ref.imag) < 1e-12, (call, got, ref)
        po = O.plaquette(g.Get(), list(dims))
        assert abs(got[0] - po[0]) < 1e-12 and abs(got[1] - po[1]) < 1e-12, (call, got, po)


def test_noalloc_plaquette_rejects_bad_enums_and_huge_dims():
    from sun_b200._native import SunLatticeParams, lib
    dummy = C.c_void_p(16)  # never dereferenced: the checks come first
    for prec, order in ((7, 0), (0, 5)):
        p = SunLatticeParams(3, (C.c_int * 4)(4, 4, 4, 4), 0.0, 0, order, prec, 0, 0)
        assert lib().sun_plaquette_noalloc(dummy, C.byref(p), dummy, None) == 1  # SUN_ERR_INVALID_ARG
    # dimensions whose product overflows 64 bits are refused, not wrapped
    p = SunLatticeParams(3, (C.c_int * 4)(2 ** 30, 2 ** 30, 2 ** 30, 2), 0.0, 0, 0, 0, 0, 0)
    assert lib().sun_plaquette_noalloc(dummy, C.byref(p), dummy, None) == 7  # SUN_ERR_CAPACITY


def test_noalloc_plaquette_allocates_nothing(ctx):
    import torch
    from sun_b200 import gauge
    from sun_b200._native import lib
    g = gauge(ctx, N=3, dims=(8, 8, 8, 8), atype=1, prec="f32", seed=4)
    g.Init(hot=True)
    p = _params(3, (8, 8, 8, 8), 1, "f32")
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    args = (C.c_void_p(g.GetPtr()), C.byref(p), C.c_void_p(out.data_ptr()), None)
    assert lib().sun_plaquette_noalloc(*args) == 0
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        assert lib().sun_plaquette_noalloc(*args) == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0


def test_noalloc_plaquette_rejects_oversized_lattice():
    from sun_b200._native import lib
    p = _params(3, (64, 64, 64, 64), 1, "f32")
    dummy = C.c_void_p(16)  # never dereferenced: the size check comes first
    assert lib().sun_plaquette_noalloc(dummy, C.byref(p), dummy, None) == 7  # SUN_ERR_CAPACITY
    assert b"exceed the fixed scratch" in lib().sun_last_error_string(None)
