"""Distribution of the SU(2) heatbath draw as the update kernels make it on
the GPU (sun_debug_su2_draws), FP32 and FP64.

The heatbath element a = (a0, a_vec) of generate_su2_matrix_milc
(include/device_PHB_OVR.h:163-223) has a0 distributed with density
sqrt(1 - a0^2) exp(alpha a0) on [-1, 1] and a_vec uniform on the sphere of
radius sqrt(1 - a0^2).  The FP32 draw runs the hardware approximations of
log, exp and sincos; these tests check it against the exact law:
  * chi^2 of a0 over 64 bins of equal exact probability, 2^21 draws,
    bound chi^2 < 63 + 6 sqrt(126) (p ~ 1e-7 for a correct draw);
  * mean of a0 against I_2(alpha) / I_1(alpha) within 5 standard errors;
  * |a| = 1, and a3 / |a_vec| and the azimuth uniform (chi^2, 32 bins);
and per draw against the oracle's FP64 restatement fed the same Philox
uniforms: FP64 to 1e-12, FP32 to 1e-4 but for accept/reject decisions
flipped at the rounding boundary (under 0.5 % of draws).
"""
import ctypes as C

import numpy as np
import pytest
from scipy.special import ive

from oracle import oracle as O

pytestmark = pytest.mark.gpu

ALPHAS = [0.3, 1.2, 2.0, 2.5, 6.0, 16.0]  # Creutz for alpha <= 2, Kennedy-Pendleton above
N_DRAWS = 1 << 21


def draws(prec, alpha, seed, n):
    from sun_b200._native import check, lib
    out = np.zeros(4 * n)
    check(lib().sun_debug_su2_draws(0 if prec == "f32" else 1, alpha, seed, n,
                                    out.ctypes.data_as(C.POINTER(C.c_double))))
    return out.reshape(n, 4)


def exact_edges(alpha, nbins):
    """Bin edges of equal probability under sqrt(1 - x^2) exp(alpha x)."""
    x = np.linspace(-1.0, 1.0, 400001)
    f = np.sqrt(np.clip(1.0 - x * x, 0.0, None)) * np.exp(alpha * (x - 1.0))
    cdf = np.concatenate([[0.0], np.cumsum(0.5 * (f[1:] + f[:-1]) * np.diff(x))])
    cdf /= cdf[-1]
    e = np.interp(np.linspace(0.0, 1.0, nbins + 1), cdf, x)
    e[0], e[-1] = -1.0 - 1e-12, 1.0 + 1e-12
    return e


def chi2_uniform_bins(counts):
    exp = counts.sum() / len(counts)
    return ((counts - exp) ** 2 / exp).sum()


@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("alpha", ALPHAS)
def test_draw_matches_exact_density(prec, alpha):
    a = draws(prec, alpha, 20261203 + int(alpha * 10), N_DRAWS)
    a0 = a[:, 0]
    counts = np.histogram(a0, exact_edges(alpha, 64))[0]
    chi2 = chi2_uniform_bins(counts)
    assert counts.sum() == N_DRAWS
    assert chi2 < 63 + 6 * np.sqrt(126), chi2
    # E[a0] = I_2(alpha) / I_1(alpha); var from the same density
    mean = ive(2, alpha) / ive(1, alpha)
    var = 1.0 - 3.0 * mean / alpha - mean * mean  # E[a0^2] = 1 - 3 E[a0] / alpha
    assert abs(a0.mean() - mean) < 5 * np.sqrt(var / N_DRAWS), (a0.mean(), mean)
    norm = np.sqrt((a * a).sum(axis=1))
    assert np.abs(norm - 1).max() < (5e-6 if prec == "f32" else 1e-13)
    r = np.sqrt(np.clip(1 - a0 * a0, 1e-300, None))
    keep = r > 1e-3
    c3 = np.histogram(a[keep, 3] / r[keep], np.linspace(-1, 1, 33))[0]
    phi = np.arctan2(a[keep, 2], a[keep, 1])
    cphi = np.histogram(phi, np.linspace(-np.pi, np.pi, 33))[0]
    assert chi2_uniform_bins(c3) < 31 + 6 * np.sqrt(62)
    assert chi2_uniform_bins(cphi) < 31 + 6 * np.sqrt(62)


@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("alpha", ALPHAS)
def test_draw_matches_oracle_per_draw(prec, alpha):
    n, seed = 2048, 77 + int(alpha * 100)
    a = draws(prec, alpha, seed, n)
    mode = O.RNG_PHILOX32 if prec == "f32" else O.RNG_PHILOX64
    ref = np.array([O.su2_generate(alpha, mode, seed, i, 0, 0)[0] for i in range(n)])
    d = np.abs(a - ref).max(axis=1)
    if prec == "f64":
        assert d.max() < 1e-12, d.max()
    else:
        assert np.mean(d > 1e-4) < 0.005, (np.mean(d > 1e-4), np.sort(d)[-5:])
