"""CPU tests of the C-ABI library: it loads, exports every function the
header declares, and its host-side scheduling rules behave."""
import ctypes as C

import pytest

from sun_b200 import _native as nat


def test_library_exports_every_header_symbol():
    L = nat.lib()
    names = nat.header_functions()
    assert len(names) >= 40
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert L.sun_version().startswith(b"sun_b200")


def test_errors_are_status_codes_not_exits():
    L = nat.lib()
    h = C.c_void_p()
    assert L.sun_lattice_create(None, None, C.byref(h)) == 1  # SUN_ERR_INVALID_ARG
    assert L.sun_plaquette(None, None, None) == 1
    assert L.sun_batch_destroy(None) == 1


def test_admission_rule_fifo_budget_and_slots():
    from sun_b200 import admit_count
    assert admit_count([10, 10, 10], budget=100, used=0, free_slots=8) == 3
    assert admit_count([10, 10, 10], budget=100, used=0, free_slots=2) == 2
    assert admit_count([50, 60, 10], budget=100, used=0, free_slots=8) == 1   # no overtaking
    assert admit_count([50, 10], budget=100, used=60, free_slots=8) == 0
    assert admit_count([], budget=100, used=0, free_slots=8) == 0
    assert admit_count([100], budget=100, used=0, free_slots=1) == 1


def test_job_footprint_scales_with_volume_and_layout():
    from sun_b200 import job_footprint, make_job
    a = job_footprint(make_job(N=3, dims=(8, 8, 8, 8), prec="f32", layout=0))
    b = job_footprint(make_job(N=3, dims=(8, 8, 8, 16), prec="f32", layout=0))
    c = job_footprint(make_job(N=3, dims=(8, 8, 8, 8), prec="f32", layout=1))
    d = job_footprint(make_job(N=3, dims=(8, 8, 8, 8), prec="f64", layout=0))
    V = 8 ** 4
    assert a >= 4 * V * 9 * 8 and c >= 4 * V * 6 * 8 and c < a < b and d > a
    w = job_footprint(make_job(N=3, dims=(8, 8, 8, 8), observables=4, R=4, T=4))
    assert w > job_footprint(make_job(N=3, dims=(8, 8, 8, 8), observables=1))


def test_struct_layouts():
    # the ctypes mirrors must match the C declarations' sizes
    assert C.sizeof(nat.SunLatticeParams) == 4 + 16 + 4 + 8 + 4 * 3 + 4 + 8 + 4 + 4  # with padding
    assert C.sizeof(nat.SunJob) % 8 == 0
