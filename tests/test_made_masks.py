"""MADE connectivity (host-only): output d depends only on inputs before d."""
import numpy as np
import pytest


@pytest.mark.parametrize("n,hidden", [(2, 8), (12, 64), (40, 512), (56, 512), (70, 96)])
def test_autoregressive_masks(pkg, n, hidden):
    m1, m2, m3 = pkg.proposal.made_masks(n, hidden)
    assert m1.shape == (hidden, n) and m2.shape == (hidden, hidden) and m3.shape == (n, hidden)
    paths = m3.astype(np.int64) @ m2 @ m1
    assert np.all(np.triu(paths) == 0)                 # no path from input i >= d to output d
    assert np.all(paths[np.tril_indices(n, -1)] > 0)   # every earlier input reaches output d


def test_envelope_calibration(pkg):
    rng = np.random.default_rng(0)
    logp = rng.normal(size=1000)
    logq = logp + rng.normal(scale=0.1, size=1000)
    log_c, deficit = pkg.proposal.calibrate_envelope(logp, logq)
    assert deficit == 0.0 and log_c >= np.max(logp - logq) - 1e-12
    log_c2, deficit2 = pkg.proposal.calibrate_envelope(logp, logq, quantile=0.5)
    assert log_c2 < log_c and deficit2 > 0.0
