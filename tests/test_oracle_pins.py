"""Pins of the CPU oracle: known answers and distribution tests (CPU only).

- Philox4x32 with 8 rounds (the streams, as the reference's R123) and 10 rounds against
  tests/golden/philox_kat.json, produced by the reference's own vendored Random123 header
  (src/third_party/Random123/philox.h) via oracle/ref_philox_kat.c.
- The project log against math.log.
- The binomial sampler with the chi-squared check of the reference's
  test/unit/cpp/test_rng.cpp:51-90 (same (n, p) grid, sample sizes and levels), and a
  goodness-of-fit test with the proper degrees of freedom over every sampler regime.
"""
import json
import math
import os

import numpy as np
import pytest
from scipy import stats

from oracle import pyoracle

HERE = os.path.dirname(os.path.abspath(__file__))


def test_philox_known_answers():
    with open(os.path.join(HERE, "golden", "philox_kat.json")) as f:
        kat = json.load(f)
    assert len(kat) >= 16
    assert {c["rounds"] for c in kat} == {8, 10}
    for c in kat:
        assert pyoracle.philox(c["ctr"], c["key"], c["rounds"]) == c["out"]


def test_philox_published_zero_vector():
    # Random123 known-answer for philox4x32_10 with zero counter and key.
    assert pyoracle.philox([0, 0, 0, 0], [0, 0], rounds=10) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]


def test_log_matches_libm():
    rng = np.random.default_rng(1)
    xs = np.concatenate([np.exp(rng.uniform(-700, 700, 20000)), rng.uniform(0, 1, 20000) + 1e-300,
                         1.0 + rng.uniform(-1e-6, 1e-6, 2000), [1.0, 2.0, 0.5, 2.3283064365386963e-10,
                                                                 5e-324, 1.7e308]])
    for x in xs:
        ref = math.log(x)
        got = pyoracle.log(x)
        assert abs(got - ref) <= 4e-16 * max(abs(ref), 1e-300) + 1e-300, (x, got, ref)


def _ref_style_pvalue(sample, t, p_test, t_test):
    """Chi-squared statistic and p-value exactly as test_rng.cpp:51-90 forms them
    (degrees of freedom = n_sample - 1)."""
    n = len(sample)
    obs = np.bincount(sample, minlength=t + 1)[: t + 1]
    k = np.arange(t + 1)
    exp = n * stats.binom.pmf(k, t_test, p_test)
    chi = float(np.sum((exp - obs) ** 2 / exp))
    return 1.0 - stats.chi2.cdf(chi, n - 1)


@pytest.mark.parametrize("t,p", [(10, 0.3), (8, 0.4)])
def test_binomial_reference_grid_accepts(t, p):
    sample = pyoracle.binom_many(12345, 0, t, p, 10000).astype(np.int64)
    assert _ref_style_pvalue(sample, t, p, t) >= 1 - 0.999


@pytest.mark.parametrize("t_test,p_test", [(10, 0.45), (15, 0.4)])
def test_binomial_reference_grid_rejects_wrong(t_test, p_test):
    sample = pyoracle.binom_many(12345, 1, 10, 0.3, 100).astype(np.int64)
    assert _ref_style_pvalue(sample, 10, p_test, t_test) <= 0.9


@pytest.mark.parametrize("n,p", [(10, 0.3), (40, 0.2), (1000, 0.3), (200, 0.93), (5000, 0.5),
                                 (1 << 20, 3e-6), (60, 0.999), (4000000000, 2e-9), (25, 0.4),
                                 (47, 0.5), (120, 0.19), (49, 0.5), (95, 0.5), (95, 0.75), (60, 0.45),
                                 (400, 0.5), (2100, 0.47), (2150, 0.47), (48, 0.999), (3, 0.13),
                                 (1, 0.5), (2, 0.71), (95, 0.0083), (1 << 30, 5e-9)])
def test_binomial_goodness_of_fit(n, p):
    """BINV below n min(p, 1-p) = 24 (down to a single trial and n p far below 1), the
    search from the mode up to 1000, BTRD above, against the exact binomial pmf."""
    m = 200000
    x = pyoracle.binom_many(777, n % 1000, n, p, m).astype(np.int64)
    mean, var = n * p, n * p * (1 - p)
    assert abs(x.mean() - mean) < 5 * math.sqrt(var / m) + 1e-12
    lo, hi = stats.binom.ppf(1e-6, n, p), stats.binom.ppf(1 - 1e-6, n, p)
    ks = np.arange(int(lo), int(hi) + 1)
    pmf = stats.binom.pmf(ks, n, p)
    keep = pmf * m >= 5
    ks, pmf = ks[keep], pmf[keep]
    obs = np.array([(x == k).sum() for k in ks])
    rest_obs = m - obs.sum()
    rest_exp = m * (1 - pmf.sum())
    chi = float(np.sum((obs - m * pmf) ** 2 / (m * pmf)))
    dof = len(ks) - 1
    if rest_exp >= 5:
        chi += (rest_obs - rest_exp) ** 2 / rest_exp
        dof += 1
    assert stats.chi2.sf(chi, dof) > 1e-4, (n, p, chi, dof)


@pytest.mark.parametrize("n,p", [(12, 0.25), (37, 0.33), (25, 0.5), (48, 0.145), (41, 0.415)])
def test_binv_large_sample(n, p):
    """The BINV search at the face-split sizes of the benchmark, 4 M draws: chi-squared over
    every outcome with expectation >= 5."""
    m = 1 << 22
    x = pyoracle.binom_many(99, n, n, p, m).astype(np.int64)
    obs = np.bincount(x, minlength=n + 1)[: n + 1]
    pmf = stats.binom.pmf(np.arange(n + 1), n, p)
    keep = pmf * m >= 5
    chi = float(np.sum((obs[keep] - m * pmf[keep]) ** 2 / (m * pmf[keep])))
    assert stats.chi2.sf(chi, int(keep.sum()) - 1) > 1e-4, (n, p, chi)


def test_binomial_edges():
    assert (pyoracle.binom_many(1, 0, 0, 0.5, 10) == 0).all()
    assert (pyoracle.binom_many(1, 0, 17, 0.0, 10) == 0).all()
    assert (pyoracle.binom_many(1, 0, 17, 1.0, 10) == 17).all()
    x = pyoracle.binom_many(1, 0, 3, 0.9999999, 1000)
    assert x.max() <= 3


@pytest.mark.parametrize("n,t1,c", [(5, 0.6, (0.145, 0.415, 0.29)), (16, 1.0, (0.355, 0.225, 0.5)),
                                    (3, 0.133, (0.145, 0.415, 0.71)), (7, 0.9, (0.0, 1.0, 0.0)),
                                    (4, 0.5, (0.2, 0.25, 1.0))])
def test_per_molecule_leave_law(n, t1, c):
    """The per-molecule leave of small counts against the multinomial it replaces: stay with
    1 - t1, face f with t1 s_f (s_f from the conditional selectors, a selector of 1 taking
    all that remain), chi-squared over every joint outcome with expectation >= 5."""
    from math import comb
    m = 400000
    k = pyoracle.leave_many(2024, n, n, t1, c, m).astype(np.int64)
    s0 = c[0]
    s1 = (1 - c[0]) * c[1]
    s2 = (1 - c[0]) * (1 - c[1]) * c[2]
    s3 = 1 - s0 - s1 - s2
    probs = [t1 * s0, t1 * s1, t1 * s2, t1 * s3, 1 - t1]
    assert (k.sum(axis=1) <= n).all()
    for f, sf in enumerate((s0, s1, s2, s3)):
        if sf == 0:
            assert (k[:, f] == 0).all()
    keys = k[:, 0] * (n + 1) ** 3 + k[:, 1] * (n + 1) ** 2 + k[:, 2] * (n + 1) + k[:, 3]
    uniq, obs = np.unique(keys, return_counts=True)
    expd = {}
    for a in range(n + 1):
        for b in range(n + 1 - a):
            for d in range(n + 1 - a - b):
                for e in range(n + 1 - a - b - d):
                    rest = n - a - b - d - e
                    pr = comb(n, a) * comb(n - a, b) * comb(n - a - b, d) * comb(n - a - b - d, e)
                    pr *= probs[0] ** a * probs[1] ** b * probs[2] ** d * probs[3] ** e * probs[4] ** rest
                    if pr > 0:
                        expd[a * (n + 1) ** 3 + b * (n + 1) ** 2 + d * (n + 1) + e] = pr
    assert set(uniq.tolist()) <= set(expd)
    ob = dict(zip(uniq.tolist(), obs.tolist()))
    big = [key for key, pr in expd.items() if pr * m >= 5]
    chi = sum((ob.get(key, 0) - m * expd[key]) ** 2 / (m * expd[key]) for key in big)
    rest_e = m * (1 - sum(expd[key] for key in big))
    rest_o = m - sum(ob.get(key, 0) for key in big)
    dof = len(big) - 1
    if rest_e >= 5:
        chi += (rest_o - rest_e) ** 2 / rest_e
        dof += 1
    assert stats.chi2.sf(chi, max(dof, 1)) > 1e-4, (chi, dof)
