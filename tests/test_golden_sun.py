"""The oracle against golden vectors of the reference built for SU(4) and
SU(6), and against its Wilson loops up to 4 x 4 for N = 3, 4, 6.

tests/golden/reference_golden_sun.npz was made by
tests/golden/make_golden_sun.py, which ran the reference's own builds
(NCOLORS = 3, 4, 6; oracle/ref/Makefile) on a B200.  The inputs are rebuilt
here by the oracle from their seeds; a sample of each is checked against the
one the reference was given.  Pinned:
  * PlaquetteCUB / OnePolyakovLoop / WilsonLoop with R = T = 4;
  * one OverRelaxation::Run pass for N = 4, 6 (overrelaxationSUN's N != 3
    path, include/device_PHB_OVR.h:557-567);
  * per link: heatBathSUN's N != 3 path (M = U F, device_PHB_OVR.h:426-441)
    with injected uniforms, including the number of uniforms it consumes;
    overrelaxationSUN; reunit_link's column Gram-Schmidt with the
    determinant phase (include/reunitlink.h:46-84).
"""
import json
import os
import sys

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden_sun as G  # noqa: E402

Z = np.load(os.path.join(HERE, "golden", "reference_golden_sun.npz"))
META = json.load(open(os.path.join(HERE, "golden", "reference_meta_sun.json")))
CONFIGS = META["configs"]
_CACHE = {}


def config(c):
    """The input configuration the reference measured (rebuilt, cached)."""
    if c["name"] not in _CACHE:
        U = G.config(c["name"], c["N"], tuple(c["dims"]), c["beta"], c["seed"], c["oracle_sweeps"])
        assert np.abs(U[::97] - Z[c["name"] + "_U_sample"]).max() < 1e-14, "rebuilt input differs"
        _CACHE[c["name"]] = U
    return _CACHE[c["name"]]


@pytest.mark.parametrize("c", CONFIGS, ids=[c["name"] for c in CONFIGS])
def test_measurements_match_reference(c):
    n, X = c["name"], c["dims"]
    U = config(c)
    assert np.abs(O.plaquette(U, X) - Z[n + "_plaquette"]).max() < 1e-14
    assert np.abs(O.polyakov(U, X) - Z[n + "_polyakov"]).max() < 1e-14
    w = O.wilson_loops(U, X, c["R"], c["T"])
    assert w.shape == Z[n + "_wilson"].shape
    assert np.abs(w - Z[n + "_wilson"]).max() < 1e-14


OR_CONFIGS = [c for c in CONFIGS if c["overrelax"]]


@pytest.mark.parametrize("c", OR_CONFIGS, ids=[c["name"] for c in OR_CONFIGS])
def test_overrelaxation_pass_matches_reference(c):
    n, X = c["name"], c["dims"]
    U = config(c).copy()
    O.sweeps(U, X, c["beta"], 0, 1, 1)
    assert np.abs(U - Z[n + "_or1"]).max() < 1e-12


LINK_CASES = [(int(k[1]), k.split("_", 1)[1]) for k in META["link_modes"]]


@pytest.mark.parametrize("N,mode", LINK_CASES, ids=[f"N{n}-{m}" for n, m in LINK_CASES])
def test_link_updates_match_reference(N, mode):
    Ul, Fl, uni, P = G.link_inputs(N)
    beta = META["link_modes"][f"n{N}_{mode}"]
    out, used = Z[f"n{N}_link_{mode}_out"], Z[f"n{N}_link_{mode}_used"]
    assert (used >= 0).all()  # no injected stream ran out in the reference
    kinds = set()
    for i in range(len(Ul)):
        if mode.startswith("hb"):
            R, k = O.heatbath_link(Ul[i], Fl[i], beta / N, O.RNG_INJECTED, inj=np.ascontiguousarray(uni[i]))
            assert k == used[i], (i, k, used[i])  # the same uniforms consumed: the same draw order
            kinds.add(k)
        elif mode == "or":
            R = O.overrelax_link(Ul[i], Fl[i])
        else:
            R = O.reunit_link(P[i])
        assert np.abs(R - out[i]).max() < 1e-13, (mode, i, np.abs(R - out[i]).max())
    if mode.startswith("hb"):
        assert len(kinds) > 1  # some draws retried: the retry paths are pinned too


def test_lowbeta_cases_reach_the_creutz_branch():
    """The first subgroup's draw of the low-beta heatbath goldens has
    alpha <= 2 (Creutz) for some links, that of the others alpha > 2
    (Kennedy-Pendleton) for all: both branches of the draw are pinned.
    alpha = beta / N |r| with r the SU(2) block (0, 1) of M = U F."""
    for N in (4, 6):
        Ul, Fl, _, _ = G.link_inputs(N)
        for mode, lo in (("hb", False), ("hb_lowbeta", True)):
            beta = META["link_modes"][f"n{N}_{mode}"]
            alphas = []
            for i in range(len(Ul)):
                M = Ul[i] @ Fl[i]
                r = np.array([M[0, 0].real + M[1, 1].real, M[0, 1].imag + M[1, 0].imag,
                              M[0, 1].real - M[1, 0].real, M[0, 0].imag - M[1, 1].imag])
                alphas.append(beta / N * np.sqrt((r ** 2).sum()))
            alphas = np.array(alphas)
            if lo:
                assert (alphas <= 2).any()
            else:
                assert (alphas > 2).all()
