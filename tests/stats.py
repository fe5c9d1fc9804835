"""Ensemble comparisons used by the statistical tests.

Per-sample means are compared by z = (m1 - m2) / sqrt(v1/n1 + v2/n2) (the
"within 3 standard errors" criterion); per-sample variances by the log ratio
with its kurtosis-corrected standard error; distributions by the two-sample
Kolmogorov-Smirnov test.  Sample instants of one trajectory ensemble are
strongly correlated, and hundreds of (instant, species) cells are tested at
once, so the family-wise thresholds are stated in each helper.
"""
import numpy as np
from scipy.stats import ks_2samp


def mean_z(m1, v1, n1, m2, v2, n2):
    m1, v1, m2, v2 = (np.asarray(x, dtype=np.float64) for x in (m1, v1, m2, v2))
    se = np.sqrt(v1 / n1 + v2 / n2)
    z = np.zeros_like(m1)
    nz = se > 0
    z[nz] = (m1[nz] - m2[nz]) / se[nz]
    z[~nz] = np.where(m1[~nz] == m2[~nz], 0.0, np.inf)
    return z


def check_means(m1, v1, n1, m2, v2, n2, *, max_frac_3se=0.02, hard=5.0):
    """At most `max_frac_3se` of the cells beyond 3 SE (about 0.3% expected
    for independent cells) and none beyond `hard` SE."""
    z = np.abs(mean_z(m1, v1, n1, m2, v2, n2))
    frac = float((z > 3).mean())
    return frac <= max_frac_3se and float(z.max()) < hard, {"frac_gt3": frac, "max_z": float(z.max())}


def var_z(a, b):
    """z of log(var a / var b) with SE^2 = (kurt_a - 1)/n_a + (kurt_b - 1)/n_b."""
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    va, vb = a.var(ddof=1), b.var(ddof=1)
    if va == 0 or vb == 0:
        return 0.0 if va == vb else np.inf
    ka = ((a - a.mean()) ** 4).mean() / va ** 2
    kb = ((b - b.mean()) ** 4).mean() / vb ** 2
    return float(np.log(va / vb) / np.sqrt((ka - 1) / len(a) + (kb - 1) / len(b)))


def ks_pvalues(A, B):
    """Two-sample KS p-values column by column ([n][cells] arrays)."""
    A = np.asarray(A).reshape(A.shape[0], -1)
    B = np.asarray(B).reshape(B.shape[0], -1)
    ps = []
    for j in range(A.shape[1]):
        if np.ptp(A[:, j]) == 0 and np.ptp(B[:, j]) == 0:
            ps.append(1.0 if A[0, j] == B[0, j] else 0.0)
        else:
            ps.append(float(ks_2samp(A[:, j], B[:, j]).pvalue))
    return np.array(ps)
