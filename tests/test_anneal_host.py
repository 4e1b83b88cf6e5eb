"""Host-side helpers of the annealer (no GPU)."""
import numpy as np

import anneal as A


def test_rank_correlation_matches_scipy():
    from scipy.stats import spearmanr
    rng = np.random.default_rng(4)
    x = rng.normal(size=200)
    y = x + rng.normal(size=200)
    y[::7] = y[0]                        # ties
    assert abs(A.rank_correlation(x, y) - spearmanr(x, y).correlation) < 1e-12
    assert A.rank_correlation(x, -x) == -1.0
