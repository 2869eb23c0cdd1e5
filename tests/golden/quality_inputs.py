"""Seeded inputs of the IGD fixtures in quality_reference.json (shared by
make_quality_golden.py and the tests)."""
import numpy as np


def approximation(seed, n, M):
    """(n, M) FP32 points near the unit sphere, some dominated, with three NaN
    rows and one infinite value (the metric drops non-finite rows)."""
    rng = np.random.default_rng(seed)
    x = rng.random((n, M)) + 0.05
    x = x / np.linalg.norm(x, axis=1, keepdims=True) * (1.0 + 0.3 * rng.random((n, 1)))
    x = x.astype(np.float32)
    x[:3] = np.nan
    x[3, 0] = np.inf
    return x
