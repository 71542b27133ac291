"""The sm_100a engine against golden vectors of the reference built for
SU(4) and SU(6), and against its Wilson loops up to 4 x 4 for N = 3, 4, 6
(tests/golden/reference_golden_sun.npz, made by running the reference's own
NCOLORS = 3, 4, 6 builds on a B200 -- tests/golden/make_golden_sun.py).

Tolerances as in the other parity tests: measurements (FP64 arithmetic)
1e-12 from FP64 links and 1e-6 from FP32-stored links; one overrelaxation
pass per link 1e-11 (FP64) and 1.2e-4 (FP32 storage and arithmetic);
reunitarization (FP64 arithmetic) 1e-13 from FP64 links.  The engine
recomputes each SU(2) block of U S^dagger for N >= 4 where the reference
keeps M = U S^dagger; the results agree to rounding.
"""
import json
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden_sun as G  # noqa: E402

Z = np.load(os.path.join(HERE, "golden", "reference_golden_sun.npz"))
META = json.load(open(os.path.join(HERE, "golden", "reference_meta_sun.json")))
CONFIGS = META["configs"]
_CACHE = {}


def config(c):
    if c["name"] not in _CACHE:
        _CACHE[c["name"]] = G.config(c["name"], c["N"], tuple(c["dims"]), c["beta"], c["seed"], c["oracle_sweeps"])
    return _CACHE[c["name"]]


def storage(N):
    out = [("f64", 0, 1e-12), ("f32", 0, 1e-6)]
    if N == 3:
        out += [("f32", 1, 1e-6), ("f64", 1, 1e-12)]
    return out


CASES = [(c, prec, lay, tol) for c in CONFIGS for prec, lay, tol in storage(c["N"])]


def _id(case):
    c, prec, lay, _ = case
    return f"{c['name']}-{prec}-{['SOA', 'SOA12', 'SOA8'][lay]}"


def _lat(ctx, c, prec, lay, evenodd=True):
    from sun_b200 import gauge
    return gauge(ctx, N=c["N"], dims=tuple(c["dims"]), beta=c["beta"], atype=lay, evenodd=evenodd, prec=prec,
                 seed=1)


@pytest.mark.parametrize("case", CASES, ids=_id)
def test_measurements_match_reference(ctx, case):
    from sun_b200 import OnePolyakovLoop, PlaquetteCUB, WilsonLoop
    c, prec, lay, tol = case
    n = c["name"]
    for evenodd in (True, False):
        g = _lat(ctx, c, prec, lay, evenodd)
        g.Set(config(c))
        p = PlaquetteCUB(g).Run()
        l = OnePolyakovLoop(g).Run()
        w = WilsonLoop(g, c["R"], c["T"])
        g.Release()
        assert np.abs(np.array([p.real, p.imag]) - Z[n + "_plaquette"]).max() < tol
        assert np.abs(np.array([l.real, l.imag]) - Z[n + "_polyakov"]).max() < tol
        assert np.abs(np.stack([w.real, w.imag], -1) - Z[n + "_wilson"]).max() < tol, (evenodd,)


OR_CONFIGS = [c for c in CONFIGS if c["overrelax"]]


@pytest.mark.parametrize("c", OR_CONFIGS, ids=[c["name"] for c in OR_CONFIGS])
@pytest.mark.parametrize("prec,tol", [("f64", 1e-11), ("f32", 1.2e-4)])
def test_overrelaxation_pass_matches_reference(ctx, c, prec, tol):
    from sun_b200 import OverRelaxation
    g = _lat(ctx, c, prec, 0)
    g.Set(config(c))
    OverRelaxation(g).Run(1)
    d = np.abs(g.Get() - Z[c["name"] + "_or1"]).max()
    g.Release()
    assert d < tol, d


@pytest.mark.parametrize("N", [4, 6])
def test_reunitarize_matches_reference_links(ctx, N):
    """The reference's reunit_link outputs for perturbed links, set into a
    lattice at the links they came from and reunitarized by the engine."""
    from sun_b200 import Reunitarize
    c = [c for c in CONFIGS if c["N"] == N and c["dims"] == [4, 4, 4, 4]][0]
    _, _, _, P = G.link_inputs(N)
    U = config(c).copy()
    pos = [(lex, mu) for lex in range(0, 256, 4) for mu in range(4)][: len(P)]
    for k, (lex, mu) in enumerate(pos):
        U[lex, mu] = P[k]
    g = _lat(ctx, c, "f64", 0)
    g.Set(U)
    Reunitarize(g).Run()
    R = g.Get()
    g.Release()
    out = Z[f"n{N}_link_reunit_out"]
    d = max(np.abs(R[lex, mu] - out[k]).max() for k, (lex, mu) in enumerate(pos))
    assert d < 1e-13, d
