"""The three update kernels give the same bits.

k_update runs one thread per half-site; k_update_rows, which the engine takes
for small lattices of N >= 4 and of SU(3) with FP64 full links, spreads each
half-site over N lanes; k_update_tile, which it takes for larger lattices of
N >= 4, runs N warps per 32 half-sites with the staple factors staged in
shared memory and the SU(2) updates streamed from it.  Every element of the
staple sum and the update goes through the same operations in all three, so
sweeps and heatbath passes with injected uniforms must agree bit for bit on
every class, shape and mode, whichever kernel the size rule picks.
The oracle parity tests therefore hold for both kernels; the overrelaxation
and injected-heatbath parity of each is also checked here directly.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

SHAPES = [(4, 4, 4, 4), (4, 6, 8, 4), (6, 6, 6, 6), (8, 8, 8, 8)]


def _classes():
    out = []
    for N in (2, 3, 4, 6):
        out += [(N, "f64", 0), (N, "f32", 0)]
    out += [(3, "f32", 1), (3, "f64", 1), (3, "f32", 2), (3, "f64", 2)]
    return out


CASES = [(N, prec, lay, dims) for (N, prec, lay) in _classes() for dims in SHAPES
         if N <= 3 or dims[0] * dims[1] * dims[2] * dims[3] <= 1296]


def _ids(c):
    N, prec, lay, dims = c
    return f"N{N}-{prec}-{['SOA', 'SOA12', 'SOA8'][lay]}-{'x'.join(map(str, dims))}"


def _context(kind):
    from sun_b200 import Context
    old = os.environ.get("SUN_B200_UPDATE_KERNEL")
    os.environ["SUN_B200_UPDATE_KERNEL"] = kind
    try:
        return Context(0)
    finally:
        if old is None:
            del os.environ["SUN_B200_UPDATE_KERNEL"]
        else:
            os.environ["SUN_B200_UPDATE_KERNEL"] = old


@pytest.fixture(scope="module")
def ctxs():
    # "tile" runs k_update_tile where it applies (N >= 4) and the size rule
    # elsewhere
    out = (_context("sites"), _context("rows"), _context("tile"))
    yield out
    for c in out:
        c.close()


BETA = {2: 2.3, 3: 5.8, 4: 10.5, 6: 25.0}


def _pair(ctxs, N, prec, lay, dims, seed, reunit_every=0):
    from sun_b200 import gauge
    out = []
    for c in ctxs:
        g = gauge(c, N=N, dims=dims, beta=BETA[N], atype=lay, evenodd=True, prec=prec, seed=seed,
                  reunit_every=reunit_every)
        g.Init(hot=True)
        out.append(g)
    return out


def _uniforms(N, dims, seed):
    V = int(np.prod(dims))
    stride = (N * (N - 1) // 2) * 86
    u = (np.random.default_rng(seed).integers(0, 2 ** 24, size=V * 4 * stride) + 1) / 2.0 ** 24  # exact in FP32
    return u, stride


@pytest.mark.parametrize("case", CASES, ids=_ids)
def test_sweeps_identical(ctxs, case):
    from sun_b200 import Sweep
    N, prec, lay, dims = case
    gs = _pair(ctxs, N, prec, lay, dims, seed=31, reunit_every=2)
    for g in gs:
        Sweep(g, 1, 4, 3)
    for g in gs[1:]:
        assert np.array_equal(gs[0].get_image(), g.get_image())
        assert gs[0].rng_state() == g.rng_state()


@pytest.mark.parametrize("case", [c for c in CASES if c[3] == (4, 6, 8, 4)], ids=_ids)
def test_injected_heatbath_identical(ctxs, case):
    import torch
    from sun_b200 import HeatBath
    N, prec, lay, dims = case
    gs = _pair(ctxs, N, prec, lay, dims, seed=8)
    u, stride = _uniforms(N, dims, 4)
    du = torch.tensor(u, dtype=torch.float64, device="cuda")
    for g in gs:
        HeatBath(g).RunInjected(du.data_ptr(), stride)
    for g in gs[1:]:
        assert np.array_equal(gs[0].get_image(), g.get_image())


EACH = [(k, N, prec, lay) for k in (0, 1, 2)
        for N, prec, lay in [(3, "f64", 0), (3, "f32", 1), (4, "f64", 0), (4, "f32", 0), (6, "f32", 0),
                             (6, "f64", 0)]
        if k < 2 or N >= 4]


@pytest.mark.parametrize("kernel,N,prec,lay", EACH,
                         ids=[f"{['sites', 'rows', 'tile'][k]}-N{N}-{p}-{['SOA', 'SOA12'][l]}" for k, N, p, l in EACH])
def test_each_kernel_matches_oracle(ctxs, kernel, N, prec, lay):
    """One overrelaxation pass, then one heatbath pass with injected
    uniforms, against the oracle per link."""
    import torch
    from sun_b200 import HeatBath, OverRelaxation, gauge
    dims = (4, 4, 4, 8)
    X = list(dims)
    U = O.hot(N, X, 5)
    O.sweeps(U, X, BETA[N], 1, 1, 2, seed=5)
    g = gauge(ctxs[kernel], N=N, dims=dims, beta=BETA[N], atype=lay, evenodd=True, prec=prec, seed=1)
    g.Set(U)
    ref = g.Get()
    OverRelaxation(g).Run(1)
    O.sweeps(ref, X, BETA[N], 0, 1, 1)
    tol = 1e-11 if prec == "f64" else 1.2e-4
    assert np.abs(g.Get() - ref).max() < tol
    ref = g.Get()
    u, stride = _uniforms(N, dims, 6)
    du = torch.tensor(u, dtype=torch.float64, device="cuda")
    HeatBath(g).RunInjected(du.data_ptr(), stride)
    for par in (0, 1):
        for mu in range(4):
            assert O.update_phase(ref, X, par, mu, 0, BETA[N], O.RNG_INJECTED, inj=u, inj_stride=stride) == 0
    d = np.abs(g.Get() - ref).reshape(int(np.prod(dims)) * 4, -1).max(axis=1)
    frac = np.mean(d > tol)
    assert frac == 0.0 if prec == "f64" else frac < 0.01, (frac, d.max())


def test_batch_graph_with_one_mode(ctxs):
    """A captured sweep of overrelaxation alone after one of heatbath and
    overrelaxation: each capture finds the tables of the modes it runs."""
    from sun_b200 import Batch, Sweep
    for c in ctxs:
        a = _pair((c,), 4, "f32", 0, (4, 4, 4, 4), seed=12)[0]
        b = _pair((c,), 4, "f32", 0, (4, 4, 4, 4), seed=12)[0]
        batch = Batch(c)
        batch.add(b)
        batch.sweep(1, 4, 1, graph=True)
        batch.sweep(0, 1, 2, graph=True)
        batch.sweep(1, 0, 1, graph=True)
        Sweep(a, 1, 4, 1)
        Sweep(a, 0, 1, 2)
        Sweep(a, 1, 0, 1)
        assert np.array_equal(a.get_image(), b.get_image())
        batch.close()


@pytest.mark.parametrize("N,dims,prec,lay", [(3, (4, 4, 4, 8), "f32", 1), (3, (8, 8, 8, 8), "f64", 0),
                                             (3, (16, 16, 16, 16), "f32", 1), (3, (8, 8, 8, 8), "f32", 0),
                                             (4, (16, 16, 16, 16), "f32", 0), (6, (12, 12, 12, 12), "f64", 0)])
def test_overlapped_phases_are_deterministic(ctx, N, dims, prec, lay):
    """Consecutive phases overlap (programmatic dependent launch); the same
    passes on the same links must still give the same bits on every run --
    a read served from a stale cache line would not.  The SU(4) and SU(6)
    cases run the tiled kernel (by size)."""
    from sun_b200 import HeatBath, OverRelaxation, Sweep, gauge
    imgs = []
    for _ in range(3):
        g = gauge(ctx, N=N, dims=dims, beta=BETA[N], atype=lay, evenodd=True, prec=prec, seed=1234)
        g.Init(hot=True)
        for _ in range(2):
            HeatBath(g).Run(1)
            OverRelaxation(g).Run(2)
        Sweep(g, 1, 4, 2)
        imgs.append(g.get_image())
        g.Release()
    assert all(np.array_equal(imgs[0], im) for im in imgs[1:])
