"""The sm_100a engine against golden vectors of the reference itself
(tests/golden/reference_golden.npz, made by running the reference's own build
on a B200 -- see tests/golden/make_golden.py), and the ensemble plaquette at
beta = 6.0 against the reference's own Monte Carlo chain.
"""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
Z = np.load(os.path.join(HERE, "golden", "reference_golden.npz"))
META = json.load(open(os.path.join(HERE, "golden", "reference_meta.json")))
CONFIGS = META["configs"]
STORAGE = [("f64", 0, 1e-12), ("f32", 0, 1e-6), ("f32", 1, 1e-6), ("f64", 1, 1e-12)]


def _lat(ctx, c, prec, lay, evenodd=True, seed=1):
    from sun_b200 import gauge
    return gauge(ctx, N=3, dims=tuple(c["dims"]), beta=c["beta"], atype=lay, evenodd=evenodd, prec=prec, seed=seed)


@pytest.mark.parametrize("c", CONFIGS, ids=[c["name"] for c in CONFIGS])
@pytest.mark.parametrize("prec,lay,tol", STORAGE)
def test_measurements_match_reference(ctx, c, prec, lay, tol):
    from sun_b200 import OnePolyakovLoop, PlaquetteCUB, WilsonLoop
    n = c["name"]
    for evenodd in (True, False):
        g = _lat(ctx, c, prec, lay, evenodd)
        g.Set(Z[n + "_U"])
        p = PlaquetteCUB(g).Run()
        l = OnePolyakovLoop(g).Run()
        w = WilsonLoop(g, c["R"], c["T"])
        assert np.abs(np.array([p.real, p.imag]) - Z[n + "_plaquette"]).max() < tol
        assert np.abs(np.array([l.real, l.imag]) - Z[n + "_polyakov"]).max() < tol
        assert np.abs(np.stack([w.real, w.imag], -1) - Z[n + "_wilson"]).max() < tol


@pytest.mark.parametrize("c", CONFIGS, ids=[c["name"] for c in CONFIGS])
def test_overrelaxation_pass_matches_reference(ctx, c):
    from sun_b200 import OverRelaxation
    n = c["name"]
    g = _lat(ctx, c, "f64", 0)
    g.Set(Z[n + "_U"])
    OverRelaxation(g).Run(1)
    assert np.abs(g.Get() - Z[n + "_or1"]).max() < 1e-11


@pytest.mark.parametrize("c", CONFIGS, ids=[c["name"] for c in CONFIGS])
def test_reunitarize_matches_reference(ctx, c):
    from sun_b200 import Reunitarize
    n = c["name"]
    g = _lat(ctx, c, "f64", 0)
    g.Set(Z[n + "_pert"])
    Reunitarize(g).Run()
    assert np.abs(g.Get() - Z[n + "_reunit"]).max() < 1e-13


def _binned(x, min_bins=20):
    """Mean and autocorrelation-corrected error: the largest standard error
    of bin means over bin sizes leaving at least min_bins bins (the binning
    plateau of a positively correlated Markov chain)."""
    x = np.asarray(x, dtype=float)
    err = x.std(ddof=1) / np.sqrt(len(x))
    b = 2
    while len(x) // b >= min_bins:
        m = x[: len(x) // b * b].reshape(-1, b).mean(axis=1)
        err = max(err, m.std(ddof=1) / np.sqrt(len(m)))
        b *= 2
    return x.mean(), err


@pytest.mark.parametrize("prec,lay", [("f64", 0), ("f32", 1)])
def test_ensemble_plaquette_agrees_with_reference_chain(ctx, prec, lay):
    """beta = 6.0 SU(3) 8^4, cold start, 200 + 2000 sweeps of 1 HB + 4 OR with
    reunitarization every 10 -- the reference's chain used cuRAND MRG32k3a,
    this one Philox, so the chains differ and only the ensemble means agree."""
    from sun_b200 import PlaquetteCUB, Sweep, gauge
    g = gauge(ctx, N=3, dims=(8, 8, 8, 8), beta=6.0, atype=lay, prec=prec, seed=20241203, reunit_every=10)
    g.Init(hot=False)
    Sweep(g, 1, 4, 200)
    ours = []
    for _ in range(2000):
        Sweep(g, 1, 4, 1)
        p = PlaquetteCUB(g).Run()
        ours.append((p.real + p.imag) / 2)
    ref = Z["ensemble_b6_8x4_plaquette"].mean(axis=1)
    m1, e1 = _binned(ours)
    m2, e2 = _binned(ref)
    assert abs(m1 - m2) < 3.5 * np.hypot(e1, e2), (m1, e1, m2, e2)
    assert e1 < 1e-3 and e2 < 1e-3
