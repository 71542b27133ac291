"""The smearing oracle against the reference's own smearing.

tests/golden/reference_smear.npz was made by tests/golden/make_golden_smear.py,
which ran the reference build (oracle/ref/Makefile -> oracle/_ref/ref_probe)
on a B200: ApplyAPEinSpace/inTime, ApplyStoutinSpace/inTime,
ApplyHYPinSpace/inTime and ApplyMultiHitSpace on thermalized SU(3)
configurations.  The fixtures hold the smeared directions only.  Further
checks pin the pieces to independent mathematics: exp(iQ) against scipy's
Pade matrix exponential in every regime of the Cayley-Hamilton formula, and
the SU(N) projection against its defining maximum.
"""
import os

import numpy as np
import pytest
import scipy.linalg as sl

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
Z = np.load(os.path.join(HERE, "golden", "reference_smear.npz"))
CASES = sorted({k[:-5] for k in Z.files if k.endswith("_args")})


def _apply(kind, U, X, a):
    A = U.copy()
    mask = O.SPACE if kind.endswith("space") else O.TIME
    if kind.startswith("ape"):
        O.ape(A, X, a[0], int(a[1]), int(a[2]), a[3], mask)
    elif kind.startswith("stout"):
        O.stout(A, X, a[0], int(a[1]), mask)
    elif kind.startswith("hyp"):
        O.hyp(A, X, (a[3], a[4], a[5]), int(a[0]), int(a[1]), a[2], mask)
    else:
        A = O.multihit_space(U, X, int(a[0]))
    return A


@pytest.mark.parametrize("case", CASES)
def test_smearing_matches_reference(case):
    name, kind = case[:5], case[6:]
    U = Z[name + "_U"]
    X = [int(v) for v in Z[name + "_dims"]]
    A = _apply(kind, U, X, Z[case + "_args"])
    dirs = slice(0, 3) if kind.endswith("space") else slice(3, 4)
    tol = 5e-14 if kind.startswith("multihit") else 1e-14
    assert np.abs(A[:, dirs] - Z[case]).max() < tol
    # the other directions are untouched
    other = slice(3, 4) if kind.endswith("space") else slice(0, 3)
    assert np.array_equal(A[:, other], U[:, other])


def _herm_traceless(rng, scale):
    M = rng.standard_normal((3, 3)) + 1j * rng.standard_normal((3, 3))
    H = 0.5 * (M + M.conj().T)
    H -= np.trace(H) / 3 * np.eye(3)
    return H * scale / np.linalg.norm(H)


@pytest.mark.parametrize("scale", [1e-4, 0.05, 0.3, 1.0, 2.5])
def test_exp_iq_matches_pade(scale):
    rng = np.random.default_rng(int(scale * 1e4))
    for _ in range(20):
        Q = _herm_traceless(rng, scale)
        assert np.abs(O.exp_iq3(Q) - sl.expm(1j * Q)).max() < 1e-13
    # near-degenerate spectra (theta series) and c0 < 0
    for Q in (np.diag([1.0, 1.0, -2.0]) * 0.4, np.diag([-1.0, -1.0, 2.0]) * 0.4,
              np.diag([1.0, 1.0 - 1e-5, -2.0 + 1e-5]) * 0.5):
        assert np.abs(O.exp_iq3(Q) - sl.expm(1j * Q)).max() < 1e-12


@pytest.mark.parametrize("N", [2, 3, 4])
def test_projection_maximises_trace(N):
    """P(Q) is in SU(N) and Re tr(P Q^dag) beats random SU(N) nearby."""
    rng = np.random.default_rng(N)
    X = [2, 2, 2, 2]
    H = O.hot(N, X, 5)
    for k in range(4):
        V = H[k, 0]
        Q = V + 0.3 * (rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N)))
        P = O.project_sun(np.eye(N), Q, 50, 0.0)
        assert np.abs(P @ P.conj().T - np.eye(N)).max() < 1e-12
        assert abs(np.linalg.det(P) - 1) < 1e-12
        best = np.trace(P @ Q.conj().T).real
        for j in range(20):
            W = O.project_sun(H[(j + 4) % len(H), j % 4], Q, 1, 0.0)  # one hit from elsewhere: not better
            assert np.trace(W @ Q.conj().T).real <= best + 1e-9


def test_multihit_changes_only_time_links_and_averages():
    X = [4, 4, 4, 4]
    U = O.hot(3, X, 8)
    O.sweeps(U, X, 6.0, 1, 1, 2, seed=8)
    M = O.multihit(U, X, 6.0, 7, 99)
    assert np.array_equal(M[:, :3], U[:, :3])
    assert not np.allclose(M[:, 3], U[:, 3])
    # a mean of 8 SU(3) matrices: |entries| <= 1, not unitary
    assert np.abs(M[:, 3]).max() <= 1 + 1e-12
    # nhit = 0 returns the input
    assert np.array_equal(O.multihit(U, X, 6.0, 0, 99), U)
