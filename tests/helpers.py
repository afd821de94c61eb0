"""Shared checks for the parity tests."""
import numpy as np

from conftest import segments_of


def compare_paths(z, count, m, ds):
    """Bit-exact comparison of traced segments with a golden path fixture; returns mismatching rays."""
    bad = []
    ref_cnt = z["ray_count"]
    for r in range(len(ref_cnt)):
        rm, rds = segments_of(z, r)
        if count[r] != ref_cnt[r] or not np.array_equal(m[r, :count[r]], rm) or not np.array_equal(ds[r, :count[r]], rds):
            bad.append(r)
    return bad


def zscores(w1a, w2a, na, w1b, w2b, nb, mask=None):
    """Per-bin z-scores of two Monte Carlo estimates given their sums of w and w^2 over histories
    (per-history contributions, FluxRecorder statistics): var(sum w) = sum w^2 - (sum w)^2 / N."""
    va = np.maximum(w2a - w1a * w1a / na, 0)
    vb = np.maximum(w2b - w1b * w1b / nb, 0)
    if mask is None:
        mask = (w1a > 0) | (w1b > 0)
    den = np.sqrt(va + vb)[mask]
    ok = den > 0
    return ((w1a - w1b)[mask][ok]) / den[ok]


def median_relative_error(stats, n):
    """Median over bins with flux of R = sqrt(sum w^2 / (sum w)^2 - 1/N) (FluxRecorder statistics)."""
    w1, w2 = stats[1], stats[2]
    m = w1 > 0
    return float(np.median(np.sqrt(np.maximum(w2[m] / w1[m] ** 2 - 1.0 / n, 0))))
