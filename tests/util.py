"""Comparison helpers used by the parity tests."""
import numpy as np

# rwig's own known-answer tolerance: 10 * sqrt(.Machine$double.eps) (test_sinkhorn.R:4)
GOLDEN_TOL = 10 * np.sqrt(np.finfo(float).eps)
# parity bar against the CPU oracle on the same inputs: relative error <= 1e-10
PARITY_TOL = 1e-10


def mean_rel_diff(target, current):
    """R's all.equal(target, current) statistic: sum|t - c| / sum|t|."""
    t = np.asarray(target, dtype=float).ravel()
    c = np.asarray(current, dtype=float).ravel()
    assert t.shape == c.shape, (t.shape, c.shape)
    den = np.abs(t).sum()
    return float(np.abs(t - c).sum() / den) if den > 0 else float(np.abs(t - c).sum())


def rel_err(x, ref, scale=None):
    """Normwise relative error max|x - ref| / max|ref| over the finite entries;
    non-finite entries must agree exactly.  `scale` replaces max|ref| as the
    denominator when given (for a dual pair (f, g), which is defined up to a
    shared constant, both use max(|f|, |g|))."""
    x = np.asarray(x, dtype=float).ravel()
    ref = np.asarray(ref, dtype=float).ravel()
    assert x.shape == ref.shape, (x.shape, ref.shape)
    fin = np.isfinite(ref)
    assert np.array_equal(np.isfinite(x), fin), "non-finite pattern differs"
    assert np.array_equal(x[~fin], ref[~fin], equal_nan=True), "non-finite values differ"
    if not fin.any():
        return 0.0
    den = np.abs(ref[fin]).max() if scale is None else scale
    num = np.abs(x[fin] - ref[fin]).max()
    return float(num / den) if den > 0 else float(num)


def dual_scale(f, g):
    v = np.concatenate([np.ravel(f), np.ravel(g)])
    v = v[np.isfinite(v)]
    return float(np.abs(v).max()) if v.size else 1.0
