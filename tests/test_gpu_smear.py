"""GPU parity of smearing and multihit (src/smear/) through the C ABI.

The engine against (a) the reference's own smearing output
(tests/golden/reference_smear.npz, SU(3) FP64) and (b) the FP64 oracle for
every N, layout, order and precision.  Tolerances per link: FP64 1e-12
(1e-11 for the 8-parameter layout, whose reconstruction divides by
|e01|^2 + |e02|^2); FP32 5e-5 per smearing step of SU(3)-valued results from
FP32-stored input, looser for the iterated projections of HYP (three
projection levels) and for multihit averages.  Heatbath multihit in FP32 may
flip an accept/reject decision at the rounding boundary, so there at least
99% of links must agree.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
Z = np.load(os.path.join(HERE, "golden", "reference_smear.npz"))
REF_CASES = sorted({k[:-5] for k in Z.files if k.endswith("_args")})


def _make(ctx, N, dims, prec="f64", lay=0, evenodd=True, beta=6.0):
    from sun_b200 import gauge
    return gauge(ctx, N=N, dims=dims, beta=beta, atype=lay, evenodd=evenodd, prec=prec, seed=3)


def _apply_gpu(kind, g, a, out=None):
    import sun_b200 as S
    if kind == "ape_space":
        S.ApplyAPEinSpace(g, a[0], int(a[1]), int(a[2]), a[3])
    elif kind == "ape_time":
        S.ApplyAPEinTime(g, a[0], int(a[1]), int(a[2]), a[3])
    elif kind == "stout_space":
        S.ApplyStoutinSpace(g, a[0], int(a[1]))
    elif kind == "stout_time":
        S.ApplyStoutinTime(g, a[0], int(a[1]))
    elif kind == "hyp_space":
        S.ApplyHYPinSpace(g, int(a[0]), int(a[1]), a[2], S.ParamHYP(a[3], a[4], a[5]))
    elif kind == "hyp_time":
        S.ApplyHYPinTime(g, int(a[0]), int(a[1]), a[2], S.ParamHYP(a[3], a[4], a[5]))
    elif kind == "multihit_space":
        S.ApplyMultiHitSpace(g, out, int(a[0]))
        return out
    return g


def _apply_oracle(kind, U, X, a):
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


@pytest.mark.parametrize("evenodd", [False, True], ids=["normal", "evenodd"])
@pytest.mark.parametrize("case", REF_CASES)
def test_smearing_matches_reference(ctx, case, evenodd):
    """The engine's FP64 smearing against the reference's own output."""
    name, kind = case[:5], case[6:]
    U = Z[name + "_U"]
    dims = tuple(int(v) for v in Z[name + "_dims"])
    g = _make(ctx, 3, dims, "f64", 0, evenodd)
    g.Set(U)
    out = None
    if kind.startswith("multihit"):
        out = _make(ctx, 3, dims, "f64", 0, evenodd)
    r = _apply_gpu(kind, g, Z[case + "_args"], out).Get()
    dirs = slice(0, 3) if kind.endswith("space") else slice(3, 4)
    other = slice(3, 4) if kind.endswith("space") else slice(0, 3)
    tol = 5e-14 if kind.startswith("multihit") else 1e-13
    assert np.abs(r[:, dirs] - Z[case]).max() < tol
    assert np.abs(r[:, other] - U[:, other]).max() < 1e-15


SMEAR = [  # kind, args
    ("ape_space", (0.2, 2, 10, 1e-10)),
    ("ape_time", (0.25, 1, 8, 1e-10)),
    ("stout_space", (0.1, 2)),
    ("stout_time", (0.15, 1)),
    ("hyp_space", (1, 8, 1e-10, 0.75, 0.6, 0.3)),
    ("hyp_time", (1, 8, 1e-10, 0.75, 0.6, 0.3)),
    ("multihit_space", (4,)),
]
CLASSES = [  # N, prec, layout, evenodd
    (3, "f64", 0, True), (3, "f64", 0, False), (3, "f32", 1, True), (3, "f64", 1, False),
    (3, "f32", 2, True), (3, "f64", 2, True), (2, "f64", 0, True), (4, "f64", 0, False), (4, "f32", 0, True),
]


def _tol(kind, prec, lay, steps):
    if prec == "f64":
        return 1e-11 if lay == 2 else 1e-12
    base = 5e-4 if lay == 2 else 5e-5
    if kind.startswith("hyp"):
        base *= 4
    if kind.startswith("multihit"):
        base *= 4
    return base * max(1, steps)


def _cid(c):
    N, prec, lay, eo = c
    return f"N{N}-{prec}-{['SOA', 'SOA12', 'SOA8'][lay]}-{'eo' if eo else 'lex'}"


@pytest.mark.parametrize("cls", CLASSES, ids=_cid)
@pytest.mark.parametrize("kind,args", SMEAR, ids=[k for k, _ in SMEAR])
def test_smearing_matches_oracle(ctx, kind, args, cls):
    N, prec, lay, eo = cls
    if kind.startswith("stout") and N != 3:
        pytest.skip("stout smearing is SU(3) only")
    dims = (4, 4, 4, 6)
    beta = {2: 2.3, 3: 5.8, 4: 10.5}[N]
    U = O.hot(N, list(dims), 31)
    O.sweeps(U, list(dims), beta, 1, 1, 2, seed=31)
    g = _make(ctx, N, dims, prec, lay, eo, beta)
    g.Set(U)
    Us = g.Get()  # the stored (rounded / reconstructed) input
    out = _make(ctx, N, dims, prec, 0, eo, beta) if kind.startswith("multihit") else None
    r = _apply_gpu(kind, g, args, out).Get()
    ref = _apply_oracle(kind, Us, list(dims), args)
    steps = 1 if kind.startswith("multihit") else int(args[1] if kind[:3] in ("ape", "sto") else args[0])
    assert np.abs(r - ref).max() < _tol(kind, prec, lay, steps)
    if not kind.startswith("multihit"):
        # FP32 8-parameter storage rebuilds 5 entries through a 1/n division
        utol = 1e-12 if prec == "f64" else (1e-4 if lay == 2 else 2e-5)
        assert O.unitarity_violation(r, list(dims)) < utol


@pytest.mark.parametrize("cls", [(3, "f64", 0, True), (3, "f64", 1, False), (2, "f64", 0, True),
                                 (4, "f64", 0, True), (3, "f32", 1, True)], ids=_cid)
def test_multihit_matches_oracle(ctx, cls):
    N, prec, lay, eo = cls
    import sun_b200 as S
    dims = (4, 4, 4, 4)
    beta = {2: 2.3, 3: 5.8, 4: 10.5}[N]
    U = O.hot(N, list(dims), 41)
    O.sweeps(U, list(dims), beta, 1, 1, 2, seed=41)
    g = _make(ctx, N, dims, prec, lay, eo, beta)
    g.Set(U)
    Us = g.Get()
    out = _make(ctx, N, dims, prec, 0, eo, beta)
    S.ApplyMultiHit(g, out, 777, 6)
    r = out.Get()
    mode = O.RNG_PHILOX64 if prec == "f64" else O.RNG_PHILOX32
    ref = O.multihit(Us, list(dims), beta, 6, 777, mode)
    assert np.abs(r[:, :3] - Us[:, :3]).max() < 1e-15
    d = np.abs(r[:, 3] - ref[:, 3]).reshape(len(r), -1).max(axis=1)
    if prec == "f64":
        assert d.max() < 1e-11
    else:
        assert np.mean(d < 2e-4) >= 0.99


def test_smearing_argument_errors(ctx):
    import sun_b200 as S
    from sun_b200._native import SunError, lib
    g4 = _make(ctx, 4, (4, 4, 4, 4))
    g4.Init(hot=True)
    with pytest.raises(SunError):
        S.ApplyStoutinSpace(g4, 0.1, 1)
    g3 = _make(ctx, 3, (4, 4, 4, 4))
    g3.Init(hot=True)
    assert lib().sun_smear_ape(g3.h, 0.1, 1, 5, 0.0, 0, None) != 0      # empty direction mask
    assert lib().sun_smear_ape(g3.h, 0.1, 1, 5, 0.0, 16, None) != 0     # no such direction
    o12 = _make(ctx, 3, (4, 4, 4, 4), "f64", 1)
    with pytest.raises(SunError):
        S.ApplyMultiHit(g3, o12, 1, 2)                                 # averages need SOA
    with pytest.raises(SunError):
        S.ApplyMultiHit(g3, g3, 1, 2)                                  # in place is refused
    # steps = 0 leaves the field alone
    before = g3.Get()
    S.ApplyAPEinSpace(g3, 0.2, 0, 10, 0.0)
    assert np.array_equal(g3.Get(), before)


def test_smeared_wilson_loops_grow(ctx):
    """APE smearing of the spatial links increases the ground-state overlap:
    the smeared W(R, T) of a thermalized configuration exceeds the unsmeared."""
    import sun_b200 as S
    dims = (6, 6, 6, 8)
    U = O.hot(3, list(dims), 51)
    O.sweeps(U, list(dims), 6.0, 1, 2, 6, seed=51)
    g = _make(ctx, 3, dims, "f64", 0, True)
    g.Set(U)
    w0 = S.WilsonLoop(g, 2, 3).real
    S.ApplyAPEinSpace(g, 0.2, 10, 10, 1e-10)
    w1 = S.WilsonLoop(g, 2, 3).real
    assert w1[2, 3] > w0[2, 3]
    ref = U.copy()
    O.ape(ref, list(dims), 0.2, 10, 10, 1e-10, O.SPACE)
    assert np.abs(O.wilson_loops(ref, list(dims), 2, 3)[..., 0] - w1).max() < 1e-11
