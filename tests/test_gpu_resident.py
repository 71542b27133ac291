"""Resident sweeps: sun_sweep_measure of a small lattice in one cooperative
launch, grid barriers in place of the launch boundaries.

The resident path must give the launched path's bits: the same links, RNG
counters and per-sweep plaquette and Polyakov values, for one thread per
half-site and for the row-split update, with heatbath, overrelaxation and
the reunitarization schedule inside the launch.  Each grid barrier wait is
bounded; a test makes one CTA leave without arriving and checks that the
call reports the ran-out wait and that the context keeps working.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BETA = {2: 2.3, 3: 6.0, 4: 10.5}
# (N, dims, prec, layout, hot, reunit_every, n_hb, n_or, kernel)
CASES = [(3, (8, 8, 8, 8), "f64", 0, False, 0, 1, 4, "auto"),
         (3, (8, 8, 8, 8), "f64", 0, True, 3, 1, 4, "sites"),
         (3, (8, 8, 8, 8), "f32", 1, True, 2, 1, 4, "auto"),
         (3, (4, 6, 4, 8), "f32", 2, True, 0, 2, 1, "auto"),
         (2, (8, 8, 8, 8), "f32", 0, True, 2, 1, 3, "auto"),
         (4, (6, 6, 6, 6), "f64", 0, True, 4, 1, 2, "auto"),
         (4, (4, 4, 4, 8), "f32", 0, True, 0, 0, 3, "auto"),
         (3, (6, 6, 6, 6), "f64", 0, True, 0, 3, 0, "rows")]


def _ids(c):
    N, dims, prec, lay, hot, re, nh, no, k = c
    return f"N{N}-{'x'.join(map(str, dims))}-{prec}-{['SOA', 'SOA12', 'SOA8'][lay]}-hb{nh}or{no}-{k}"


def _context(**env):
    from sun_b200 import Context
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        return Context(0)
    finally:
        for k, v in old.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v


def _lattice(ctx, c, seed=21):
    from sun_b200 import gauge
    N, dims, prec, lay, hot, re, _, _, _ = c
    g = gauge(ctx, N=N, dims=dims, beta=BETA[N], atype=lay, evenodd=True, prec=prec, seed=seed, reunit_every=re)
    g.Init(hot=hot)
    return g


def _runs_resident(ctx, c):
    """True when sun_sweep_measure takes the resident path for this case: a
    CTA told to skip its first barrier makes the call fail."""
    from sun_b200 import SweepMeasure
    from sun_b200._native import SunError, lib
    g = _lattice(ctx, c, seed=5)
    assert lib().sun_debug_resident_barrier(ctx.h, 2_000_000, 0) == 0
    try:
        SweepMeasure(g, c[6], c[7], 1)
        took = False
    except SunError as e:
        assert "ran out" in str(e)
        took = True
    finally:
        assert lib().sun_debug_resident_barrier(ctx.h, 0, -1) == 0
    g.Release()
    return took


@pytest.mark.parametrize("case", CASES, ids=_ids)
def test_resident_sweeps_match_launched_path(case):
    from sun_b200 import SweepMeasure
    kernel = case[-1]
    env = {} if kernel == "auto" else {"SUN_B200_UPDATE_KERNEL": kernel}
    on = _context(SUN_B200_RESIDENT="1", **env)
    off = _context(SUN_B200_RESIDENT="0", **env)
    try:
        assert _runs_resident(on, case)
        assert not _runs_resident(off, case)
        a, b = _lattice(on, case), _lattice(off, case)
        n = 7
        pa, la = SweepMeasure(a, case[6], case[7], n)
        pb, lb = SweepMeasure(b, case[6], case[7], n)
        assert np.array_equal(pa, pb) and np.array_equal(la, lb)
        assert np.array_equal(a.get_image(), b.get_image())
        assert a.rng_state() == b.rng_state()
        # a second call continues from the advanced counters
        pa, la = SweepMeasure(a, case[6], case[7], 3)
        pb, lb = SweepMeasure(b, case[6], case[7], 3)
        assert np.array_equal(pa, pb) and np.array_equal(la, lb)
        assert np.array_equal(a.get_image(), b.get_image())
        assert a.rng_state() == b.rng_state()
        a.Release()
        b.Release()
    finally:
        on.close()
        off.close()


def test_resident_calls_longer_than_one_launch():
    """300 sweeps take two resident launches (256 sweeps at most each): the
    second continues from the first's counters, with the launched path's
    links and per-sweep values."""
    from sun_b200 import SweepMeasure
    case = CASES[2]
    on = _context(SUN_B200_RESIDENT="1")
    off = _context(SUN_B200_RESIDENT="0")
    try:
        a, b = _lattice(on, case), _lattice(off, case)
        pa, la = SweepMeasure(a, 1, 4, 300)
        pb, lb = SweepMeasure(b, 1, 4, 300)
        assert np.array_equal(pa, pb) and np.array_equal(la, lb)
        assert np.array_equal(a.get_image(), b.get_image())
        assert a.rng_state() == b.rng_state()
        a.Release()
        b.Release()
    finally:
        on.close()
        off.close()


def test_resident_barrier_wait_runs_out_and_context_recovers():
    from sun_b200 import PlaquetteCUB, SweepMeasure
    from sun_b200._native import SunError, lib
    ctx = _context(SUN_B200_RESIDENT="1")
    try:
        c = CASES[0]
        g = _lattice(ctx, c)
        assert lib().sun_debug_resident_barrier(ctx.h, 1_000_000, 3) == 0
        with pytest.raises(SunError) as ei:
            SweepMeasure(g, 1, 4, 2)
        assert ei.value.status == 8 and "ran out" in str(ei.value)  # SUN_ERR_DEVICE_FLAG
        assert lib().sun_debug_resident_barrier(ctx.h, 0, -1) == 0
        # the context and a fresh lattice work; the failed one can be restarted
        h = _lattice(ctx, c, seed=6)
        p, l = SweepMeasure(h, 1, 4, 2)
        assert np.all(np.isfinite(p)) and 0.0 < p[-1, 0] < 1.0
        g.Init(hot=False)
        SweepMeasure(g, 1, 4, 1)
        assert 0.0 < PlaquetteCUB(g).Run().real < 1.0
    finally:
        ctx.close()
