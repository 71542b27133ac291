"""sun_sweep_measure: n sweeps with the plaquette and the Polyakov loop after
each, in one call -- the same links, RNG counters and per-sweep values as
sun_sweep + sun_plaquette + sun_polyakov called sweep by sweep, and the last
values as the oracle's on the final configuration (1e-12)."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

CASES = [(3, (8, 8, 8, 8), "f64", 0), (3, (4, 4, 4, 8), "f32", 1), (4, (4, 4, 4, 4), "f32", 0),
         (6, (4, 4, 4, 4), "f64", 0)]
BETA = {3: 6.0, 4: 10.5, 6: 25.0}


@pytest.mark.parametrize("case", CASES, ids=[f"N{c[0]}-{'x'.join(map(str, c[1]))}-{c[2]}" for c in CASES])
def test_sweep_measure_matches_sweep_by_sweep_calls(ctx, case):
    from sun_b200 import OnePolyakovLoop, PlaquetteCUB, Sweep, SweepMeasure, gauge
    N, dims, prec, lay = case
    a, b = (gauge(ctx, N=N, dims=dims, beta=BETA[N], atype=lay, evenodd=True, prec=prec, seed=99, reunit_every=3)
            for _ in range(2))
    a.Init(hot=False)
    b.Init(hot=False)
    n = 5
    pa, la = SweepMeasure(a, 1, 4, n)
    for i in range(n):
        Sweep(b, 1, 4, 1)
        p, l = PlaquetteCUB(b).Run(), OnePolyakovLoop(b).Run()
        assert pa[i, 0] == p.real and pa[i, 1] == p.imag and la[i] == l, i
    assert np.array_equal(a.get_image(), b.get_image())
    assert a.rng_state() == b.rng_state()
    X = list(dims)
    U = a.Get()
    po, lo = O.plaquette(U, X), O.polyakov(U, X)
    assert abs(pa[-1, 0] - po[0]) < 1e-12 and abs(pa[-1, 1] - po[1]) < 1e-12
    assert abs(la[-1] - (lo[0] + 1j * lo[1])) < 1e-12


def test_captured_measurements_keep_their_partials():
    """The captured sweep-and-measure graph (resident sweeps off) replayed
    after Wilson loops up to 4x4, which need more CTA partials than the
    graph's measurements: the replays still give the sweep-by-sweep values."""
    import os
    from sun_b200 import Context, OnePolyakovLoop, PlaquetteCUB, Sweep, SweepMeasure, WilsonLoop, gauge
    old = os.environ.get("SUN_B200_RESIDENT")
    os.environ["SUN_B200_RESIDENT"] = "0"
    try:
        c = Context(0)
    finally:
        if old is None:
            del os.environ["SUN_B200_RESIDENT"]
        else:
            os.environ["SUN_B200_RESIDENT"] = old
    try:
        a, b = (gauge(c, N=3, dims=(8, 8, 8, 8), beta=6.0, atype=0, evenodd=True, prec="f64", seed=17)
                for _ in range(2))
        a.Init(hot=True)
        b.Init(hot=True)
        SweepMeasure(a, 1, 4, 2)
        Sweep(b, 1, 4, 2)
        wa, wb = WilsonLoop(a, 4, 4), WilsonLoop(b, 4, 4)
        assert np.array_equal(wa, wb)
        pa, la = SweepMeasure(a, 1, 4, 3)
        for i in range(3):
            Sweep(b, 1, 4, 1)
            p, l = PlaquetteCUB(b).Run(), OnePolyakovLoop(b).Run()
            assert pa[i, 0] == p.real and pa[i, 1] == p.imag and la[i] == l, i
        assert np.array_equal(a.get_image(), b.get_image())
    finally:
        c.close()
