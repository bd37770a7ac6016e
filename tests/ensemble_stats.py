"""Two-ensemble comparison used by the statistical parity tests.

Trajectory parity with the reference solvers is statistical (their Philox stream is one
serial stream per rank, so sample paths depend on event order): two independent
ensembles of the same configuration must agree, at every record and for every observed
column, in
  * mean:      z = |m_a - m_b| / sqrt(v_a / n_a + v_b / n_b);
  * variance:  z = |v_a - v_b| / sqrt(se_a^2 + se_b^2), se^2 = (mu4 - (n-3)/(n-1) v^2) / n
               (the standard error of a sample variance from the fourth central moment);
  * distribution: the two-sample Kolmogorov-Smirnov p-value.
A trajectory is many tests (records x columns), so each criterion is applied family-wise
(Bonferroni): a z is accepted up to the cut whose two-sided tail, times the number of
tests, equals the tail of a single 3-sigma test (0.27%); a KS p-value must exceed
alpha = 0.01 divided by the number of tests.  The whole family of tests therefore has
the false-alarm probability of one 3-sigma (or one p > 0.01) test.  The uncorrected
largest z and smallest p are reported beside the verdict.
Records where both ensembles are constant (the deterministic initial state) are skipped.
"""
from __future__ import annotations

import numpy as np


def _moments(x):
    n = x.shape[0]
    m = x.mean(axis=0)
    d = x - m
    v = (d * d).sum(axis=0) / (n - 1)
    mu4 = (d ** 4).mean(axis=0)
    se2 = np.maximum(mu4 - (n - 3.0) / (n - 1.0) * v * v, 0.0) / n
    return m, v, se2


def compare(a, b, nsig=3.0, alpha=0.01, cols=None):
    """a, b: arrays [member][record][column].  Returns a report dict; report['ok'] is the
    verdict and report['worst'] names the worst record/column of each criterion."""
    from scipy.stats import ks_2samp

    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if cols is not None:
        a, b = a[:, :, cols], b[:, :, cols]
    na, nb = a.shape[0], b.shape[0]
    ma, va, sa = _moments(a)
    mb, vb, sb = _moments(b)
    live = (va > 0) | (vb > 0)
    zmean = np.where(live, np.abs(ma - mb) / np.sqrt(np.maximum(va / na + vb / nb, 1e-300)), 0.0)
    zvar = np.where(live, np.abs(va - vb) / np.sqrt(np.maximum(sa + sb, 1e-300)), 0.0)
    nrec, ncol = live.shape
    pks = np.ones((nrec, ncol))
    for r in range(nrec):
        for c in range(ncol):
            if live[r, c]:
                pks[r, c] = ks_2samp(a[:, r, c], b[:, r, c]).pvalue
    from scipy.stats import norm

    nks = int(live.sum())
    ks_cut = alpha / max(nks, 1)
    z_cut = float(norm.isf(2.0 * norm.sf(nsig) / max(nks, 1) / 2.0))
    im = np.unravel_index(np.argmax(zmean), zmean.shape)
    iv = np.unravel_index(np.argmax(zvar), zvar.shape)
    ip = np.unravel_index(np.argmin(pks), pks.shape)
    return {
        "ok": bool(zmean.max() <= z_cut and zvar.max() <= z_cut and pks.min() > ks_cut),
        "max_z_mean": float(zmean.max()), "max_z_var": float(zvar.max()), "z_cut": z_cut,
        "min_ks_p": float(pks.min()), "ks_cut": ks_cut, "n_tests": nks,
        "frac_ks_below_alpha": float((pks[live] < alpha).mean()) if nks else 0.0,
        "worst": {"mean": tuple(int(i) for i in im), "var": tuple(int(i) for i in iv),
                  "ks": tuple(int(i) for i in ip)},
        "n": (na, nb),
    }
