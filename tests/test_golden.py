"""The oracle against golden vectors produced by the reference itself.

tests/golden/reference_golden.npz was made by tests/golden/make_golden.py,
which ran the reference's own build (oracle/ref/Makefile -> oracle/_ref/) on
a B200: PlaquetteCUB / OnePolyakovLoop / WilsonLoop on fixed configurations,
one OverRelaxation::Run pass, Reunitarize::Run, and the per-link device
functions heatBathSUN (injected uniforms), overrelaxationSUN, reunit_link.
These tests pin the FP64 CPU restatement to them.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
Z = np.load(os.path.join(HERE, "golden", "reference_golden.npz"))
META = json.load(open(os.path.join(HERE, "golden", "reference_meta.json")))
CONFIGS = META["configs"]


@pytest.mark.parametrize("c", CONFIGS, ids=[c["name"] for c in CONFIGS])
def test_measurements_match_reference(c):
    n, X = c["name"], c["dims"]
    U = Z[n + "_U"]
    assert np.abs(O.plaquette(U, X) - Z[n + "_plaquette"]).max() < 1e-14
    assert np.abs(O.polyakov(U, X) - Z[n + "_polyakov"]).max() < 1e-14
    assert np.abs(O.wilson_loops(U, X, c["R"], c["T"]) - Z[n + "_wilson"]).max() < 1e-14


@pytest.mark.parametrize("c", CONFIGS, ids=[c["name"] for c in CONFIGS])
def test_overrelaxation_pass_matches_reference(c):
    n, X = c["name"], c["dims"]
    U = Z[n + "_U"].copy()
    O.sweeps(U, X, c["beta"], 0, 1, 1)
    assert np.abs(U - Z[n + "_or1"]).max() < 1e-12


@pytest.mark.parametrize("c", CONFIGS, ids=[c["name"] for c in CONFIGS])
def test_reunitarize_matches_reference(c):
    n, X = c["name"], c["dims"]
    P = Z[n + "_pert"].copy()
    O.reunitarize(P, X)
    assert np.abs(P - Z[n + "_reunit"]).max() < 1e-14


@pytest.mark.parametrize("mode", ["hb", "hb_lowbeta", "or", "reunit"])
def test_link_updates_match_reference(mode):
    Uin, Uout, used = Z[f"link_{mode}_in"], Z[f"link_{mode}_out"], Z[f"link_{mode}_used"]
    F, uni, beta = Z["link_F"], Z["link_uniforms"], float(Z[f"link_{mode}_beta"])
    for i in range(len(Uin)):
        if mode.startswith("hb"):
            R, k = O.heatbath_link(Uin[i], F[i], beta / 3, O.RNG_INJECTED, inj=np.ascontiguousarray(uni[i]))
            assert k == used[i]  # the same number of uniforms consumed: same draw order
        elif mode == "or":
            R = O.overrelax_link(Uin[i], F[i])
        else:
            R = O.reunit_link(Uin[i])
        assert np.abs(R - Uout[i]).max() < 1e-13, (mode, i)


def test_reference_files_read_by_oracle_and_written_identically(tmp_path):
    c = CONFIGS[2]
    n, X = c["name"], c["dims"]
    f = str(tmp_path / "a.bin")
    assert O.save_bin(Z[n + "_U"], X, c["beta"], f) == 0
    rc, V, g, beta = O.load_bin(3, X, f)
    assert rc == 0 and g == X and beta == c["beta"] and np.array_equal(V, Z[n + "_U"])


def test_reference_ensemble_plaquette_is_confined_phase_value():
    p = Z["ensemble_b6_8x4_plaquette"].mean(axis=1)
    assert len(p) == META["ensemble"]["meas"]
    assert 0.590 < p.mean() < 0.598
