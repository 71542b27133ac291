"""CPU tests of the FP64 oracle: known-answer vectors, algebraic identities,
layouts, gauge invariance and the heatbath distribution."""
import os

import numpy as np
import pytest

from oracle import oracle as O

X44 = [4, 4, 4, 4]


# -- Philox4x32-10 known-answer vectors (Random123 specification, kat_vectors)
@pytest.mark.parametrize("ctr,key,expect", [
    ([0, 0, 0, 0], [0, 0], [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]),
    ([0xffffffff] * 4, [0xffffffff] * 2, [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]),
    ([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0],
     [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]),
])
def test_philox_kat(ctr, key, expect):
    assert O.philox4x32_10(ctr, key) == expect


def test_uniform_streams():
    u32 = O.uniforms(1234, 17, 2, 4000, fp64=False)
    assert u32.min() > 0 and u32.max() <= 1
    k = u32 * 2 ** 24
    assert np.all(k == np.round(k))  # FP32 uniforms are exact multiples of 2^-24
    u64 = O.uniforms(1234, 17, 2, 4000, fp64=True)
    assert u64.min() > 0 and u64.max() <= 1
    assert abs(u64.mean() - 0.5) < 0.02 and abs(u32.mean() - 0.5) < 0.02
    # the first FP32 uniform is word 0 of Philox(ctr=(0, lex, mu, pass), key=seed)
    w = O.philox4x32_10([0, 17, 2, 0], [1234, 0])
    assert u32[0] == ((w[0] >> 8) + 1) / 2 ** 24
    assert u32[4] == ((O.philox4x32_10([1, 17, 2, 0], [1234, 0])[0] >> 8) + 1) / 2 ** 24


def test_su2_index_order():
    assert [O.su2_index(2, b) for b in range(1)] == [(0, 1)]
    assert [O.su2_index(3, b) for b in range(3)] == [(0, 1), (1, 2), (0, 2)]
    assert [O.su2_index(4, b) for b in range(6)] == [(0, 1), (1, 2), (2, 3), (0, 2), (1, 3), (0, 3)]
    six = [O.su2_index(6, b) for b in range(15)]
    assert six[:5] == [(i, i + 1) for i in range(5)] and six[-1] == (0, 5) and len(set(six)) == 15


@pytest.mark.parametrize("N", [2, 3, 4, 6])
def test_hot_start_special_unitary(N):
    U = O.hot(N, X44, 99)
    assert O.unitarity_violation(U, X44) < 1e-13
    d = np.linalg.det(U.reshape(-1, N, N))
    assert np.abs(d - 1).max() < 1e-13


def test_haar_moments():
    X = [8, 8, 4, 4]
    for N in (2, 3):
        U = O.hot(N, X, 7).reshape(-1, N, N)
        tr = np.trace(U, axis1=1, axis2=2)
        assert abs(np.mean(np.abs(tr) ** 2) - 1.0) < 0.05      # Haar: E|tr U|^2 = 1
        assert abs(np.mean(tr)) < 0.05
        assert abs(np.mean(np.abs(U[:, 0, 0]) ** 2) - 1.0 / N) < 0.02


@pytest.mark.parametrize("N", [2, 3, 4])
def test_cold_observables(N):
    U = O.cold(N, X44)
    assert np.allclose(O.plaquette(U, X44), [1, 1])
    assert np.allclose(O.polyakov(U, X44), [1, 0])
    assert np.allclose(O.wilson_loops(U, X44, 2, 3)[..., 0], 1)


def _gauge_transform(U, X, N, seed):
    G = O.hot(N, X, seed)[:, 0]  # one SU(N) matrix per site
    V = O.volume(X)
    Ut = np.empty_like(U)
    x = np.arange(V)
    coords = [x % X[0], (x // X[0]) % X[1], (x // (X[0] * X[1])) % X[2], x // (X[0] * X[1] * X[2])]
    for mu in range(4):
        c = [a.copy() for a in coords]
        c[mu] = (c[mu] + 1) % X[mu]
        xp = ((c[3] * X[2] + c[2]) * X[1] + c[1]) * X[0] + c[0]
        Ut[:, mu] = G @ U[:, mu] @ np.conj(np.transpose(G[xp], (0, 2, 1)))
    return Ut


@pytest.mark.parametrize("N", [2, 3, 4])
def test_gauge_invariance(N):
    X = [4, 4, 4, 6]
    U = O.hot(N, X, 5)
    Ut = _gauge_transform(U, X, N, 77)
    assert np.allclose(O.plaquette(U, X), O.plaquette(Ut, X), atol=1e-12)
    assert np.allclose(O.polyakov(U, X), O.polyakov(Ut, X), atol=1e-12)
    assert np.allclose(O.wilson_loops(U, X, 2, 2), O.wilson_loops(Ut, X, 2, 2), atol=1e-12)


def test_wilson_loop_edges_match_plaquette():
    X = [4, 4, 4, 4]
    U = O.hot(3, X, 3)
    O.sweeps(U, X, 6.0, 1, 2, 2, seed=3)
    W = O.wilson_loops(U, X, 2, 2)
    assert np.allclose(W[0, :, 0], 1) and np.allclose(W[:, 0, 0], 1)
    # W(1,1) = temporal plaquette
    assert abs(W[1, 1, 0] - O.plaquette(U, X)[1]) < 1e-12


def _ref_eo_coords(X, idd, parity):
    # Index_4D_EO (include/index.h:133-144), written out in Python
    za = idd // (X[0] // 2)
    zb = za // X[1]
    x1 = za - zb * X[1]
    x3 = zb // X[2]
    x2 = zb - x3 * X[2]
    xodd = (x1 + x2 + x3 + parity) & 1
    x0 = (2 * idd + xodd) - za * X[0]
    return x0, x1, x2, x3


def test_evenodd_image_addressing():
    X = [4, 6, 2, 4]
    V = O.volume(X)
    U = O.empty(3, X)
    for lex in range(V):
        for mu in range(4):
            U[lex, mu, 0, 0] = lex + 1j * mu
    img = O.pack(U, X, O.SOA, evenodd=True, fp64=True)
    for parity in (0, 1):
        for idd in range(V // 2):
            x = _ref_eo_coords(X, idd, parity)
            assert (sum(x) & 1) == parity
            lex = ((x[3] * X[2] + x[2]) * X[1] + x[1]) * X[0] + x[0]
            for mu in range(4):
                assert img[idd + parity * V // 2 + mu * V] == lex + 1j * mu


@pytest.mark.parametrize("layout", [O.SOA, O.SOA12, O.SOA8])
@pytest.mark.parametrize("evenodd", [True, False])
@pytest.mark.parametrize("fp64", [True, False])
def test_pack_unpack_roundtrip(layout, evenodd, fp64):
    U = O.hot(3, X44, 11)
    back = O.unpack(O.pack(U, X44, layout, evenodd, fp64), 3, X44, layout, evenodd)
    tol = 1e-12 if fp64 else 2e-6
    assert np.abs(back - U).max() < tol


def test_reunit_restores_unitarity():
    for N in (2, 3, 4, 6):
        U = O.hot(N, X44, 21)
        rng = np.random.default_rng(0)
        P = U + 1e-4 * (rng.standard_normal(U.shape) + 1j * rng.standard_normal(U.shape))
        O.reunitarize(P, X44)
        assert O.unitarity_violation(P, X44) < 1e-13
        assert np.abs(np.linalg.det(P.reshape(-1, N, N)) - 1).max() < 1e-13
        assert np.abs(P - U).max() < 1e-3


@pytest.mark.parametrize("N", [2, 3, 4])
def test_overrelaxation_is_microcanonical(N):
    X = X44
    U = O.hot(N, X, 4)
    O.sweeps(U, X, 5.0, 1, 0, 1, seed=4)
    before = U.copy()
    O.update_phase(U, X, 0, 1, 1, 5.0)
    V = O.volume(X)
    for lex in range(0, V, 7):
        x = [lex % 4, (lex // 4) % 4, (lex // 16) % 4, lex // 64]
        if sum(x) % 2:
            continue
        S = O.staple(before, X, lex, 1)
        a0 = np.trace(before[lex, 1] @ S.conj().T).real
        a1 = np.trace(U[lex, 1] @ S.conj().T).real
        assert abs(a0 - a1) < 1e-11
        assert not np.allclose(U[lex, 1], before[lex, 1])


@pytest.mark.parametrize("alpha", [0.8, 1.9, 3.0, 8.0])
def test_su2_heatbath_distribution(alpha):
    # a0 must follow sqrt(1 - a0^2) exp(alpha a0) on [-1, 1]
    n = 30000
    a0 = np.array([O.su2_generate(alpha, O.RNG_PHILOX64, seed=99, lex=i)[0][0] for i in range(n)])
    edges = np.linspace(-1, 1, 41)
    hist, _ = np.histogram(a0, edges)
    fine = np.linspace(-1, 1, 40001)
    dens = np.sqrt(np.clip(1 - fine ** 2, 0, None)) * np.exp(alpha * fine)
    cdf = np.concatenate([[0], np.cumsum((dens[1:] + dens[:-1]) / 2)])
    cdf /= cdf[-1]
    expect = n * np.diff(np.interp(edges, fine, cdf))
    m = expect > 5
    chi2 = np.sum((hist[m] - expect[m]) ** 2 / expect[m])
    dof = m.sum() - 1
    assert chi2 < dof + 5 * np.sqrt(2 * dof), (chi2, dof)


def test_heatbath_injected_matches_philox_stream():
    N = 3
    U = O.hot(N, X44, 8)
    S = O.staple(U, X44, 5, 2)
    F = S.conj().T.copy()
    u = O.uniforms(31, 5, 2, 400, fp64=True)
    A, used_a = O.heatbath_link(U[5, 2], F, 6.0 / 3, O.RNG_PHILOX64, seed=31, lex=5, mu=2)
    B, used_b = O.heatbath_link(U[5, 2], F, 6.0 / 3, O.RNG_INJECTED, inj=u)
    assert used_a == used_b > 0
    assert np.array_equal(A, B)
    _, short = O.heatbath_link(U[5, 2], F, 2.0, O.RNG_INJECTED, inj=u[:3])
    assert short == -1


def test_sweeps_thermalise_su3_beta6():
    X = X44
    U = O.cold(3, X)
    p = 0
    plaq = []
    for s in range(25):
        p = O.sweeps(U, X, 6.0, 1, 4, 1, reunit_every=5, seed=1234, pass_=p)
        plaq.append(O.plaquette(U, X).mean())
    assert p == 25
    assert 0.55 < np.mean(plaq[10:]) < 0.66
    assert O.unitarity_violation(U, X) < 1e-12


@pytest.mark.parametrize("save_fp64", [True, False])
def test_gauge_file_roundtrip(tmp_path, save_fp64):
    X = [4, 4, 2, 6]
    U = O.hot(3, X, 2)
    f = str(tmp_path / "conf.bin")
    assert O.save_bin(U, X, 6.0, f, save_fp64=save_fp64) == 0
    size = os.path.getsize(f)
    assert size == 16 + 8 + 8 + O.volume(X) * 4 * 9 * (16 if save_fp64 else 8)
    rc, V, g, beta = O.load_bin(3, X, f, save_fp64=save_fp64)
    assert rc == 0 and g == X and beta == 6.0
    assert np.abs(V - U).max() < (1e-15 if save_fp64 else 1e-6)
    # precision mismatch is refused, like ReadBin_Gauge (io_gauge.cpp:736-737)
    rc, *_ = O.load_bin(3, X, f, save_fp64=not save_fp64)
    assert rc == -3


def test_link_trace_det():
    for N in (2, 3, 4, 6):
        assert np.allclose(O.link_trace_det(O.cold(N, X44), X44), [1, 0, 1, 0])
        U = O.hot(N, X44, 8)
        t = O.link_trace_det(U, X44)
        assert abs(t[2] - 1) < 1e-13 and abs(t[3]) < 1e-13
        ref = np.trace(U.reshape(-1, N, N), axis1=1, axis2=2).mean() / N
        assert abs(t[0] - ref.real) < 1e-14 and abs(t[1] - ref.imag) < 1e-14
