"""RGS70 (n = 70, dense, rank 30) exact Born samples on one GPU by the chain rule over
the scan, rescored with the complex128 scan.

The reference samples RGS70 with a 2^35-amplitude conditional state on two GPUs; the
chain rule needs only the rank-30 scan tables.  Each sample's log p(x) from the
conditionals must equal log p(x) of its complex128 rescoring (1e-4), and the complex64
probability must match it within 1e-4 relative, the tolerance of the reference's
production manifest (FP64_probability_relative_error_max).
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_rgs70_chain_samples_rescored(pkg, fixtures):
    g = fixtures["rgs70/graph"]
    u = fixtures["rgs70/measurement_unitaries"]
    order = fixtures["rgs70/scan_order_optimized"].tolist()
    cs = pkg.ChainSampler(g, u, order, precision="c64", batch_tile=8)
    assert cs.plan.rmax == 30
    bits, p, logp = cs.sample(8, seed=70)
    del cs
    torch.cuda.empty_cache()
    so = pkg.ScanOracle(g, u, order, fp64=True, batch_tile=4)
    p128 = so.probabilities(bits)
    del so
    torch.cuda.empty_cache()
    assert np.all(p128 > 0)
    assert np.max(np.abs(p - p128) / p128) < 1e-4
    assert np.max(np.abs(logp - np.log(p128))) < 1e-4
    # Distinct strings (collisions among 8 Born samples of a 70-qubit state are vanishingly rare).
    assert len({b.tobytes() for b in bits}) == 8


def test_rgs70_searched_order_samples_are_born(pkg, fixtures):
    """256 exact samples with this package's searched order (rank 29, fused pairs): the law
    of 2^n p(x) over the samples matches the reference's 3,452 Born samples (two-sample KS
    p > 1e-3), and the linear XEB lies within 4 standard errors of the reference's pooled
    1.025; each sample's p(x) and log p(x) agree with its complex128 rescoring."""
    import json
    from pathlib import Path
    from scipy import stats

    golden = Path(__file__).resolve().parent / "golden"
    born = json.loads((golden / "rgs70_born.json").read_text())["probability_c128"]
    zref = np.concatenate([born["batch1"], born["batch2"]]) * 2.0 ** 70
    order = json.loads((golden / "searched_orders.json").read_text())["rgs70"]["order"]
    g = fixtures["rgs70/graph"]
    u = fixtures["rgs70/measurement_unitaries"]
    cs = pkg.ChainSampler(g, u, order, precision="c64", batch_tile=8)
    assert cs.plan.rmax == 29 and len(cs.plan.pairs) > 0
    bits, p, logp = cs.sample(256, seed=2029)
    del cs
    torch.cuda.empty_cache()
    z = p * 2.0 ** 70
    assert stats.ks_2samp(z, zref).pvalue > 1e-3
    se = z.std(ddof=1) / np.sqrt(len(z))
    assert abs(z.mean() - 1 - 1.025) < 4 * se
    assert np.max(np.abs(logp - np.log(p))) < 1e-4
    so = pkg.ScanOracle(g, u, fixtures["rgs70/scan_order"].tolist(), fp64=True, batch_tile=4)
    p128 = so.probabilities(bits[:16])
    del so
    torch.cuda.empty_cache()
    assert np.max(np.abs(p[:16] - p128) / p128) < 1e-4
