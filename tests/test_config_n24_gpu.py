"""The CPU-runnable configuration at full size: n = 24 random 3-regular graph, Haar SU(2)
gates, p(x) of 4096 uniform strings and 1000 exact Born samples, against the FP64 2^24
statevector (256 MiB)."""
import numpy as np
import pytest
from scipy import stats

from oracle import graph_state as gs

pytestmark = pytest.mark.gpu


def test_n24_amplitudes_and_samples(pkg):
    inst = pkg.instances.make_instance("reg3", 24, 2024, pkg.rank_profile)
    full = gs.statevector(inst.g, inst.u)
    probs = np.abs(full) ** 2
    assert abs(probs.sum() - 1.0) < 1e-10
    rng = np.random.default_rng(24)
    bits = pkg.instances.uniform_bits(4096, 24, rng)
    idx = (bits.astype(np.int64) << np.arange(24)).sum(axis=1)
    for prec, tol in (("c64", 1e-4), ("c64f32", 1e-4), ("c128", 1e-12)):
        p = pkg.ScanOracle(inst.g, inst.u, inst.order, precision=prec).probabilities(bits)
        rel = np.abs(p - probs[idx]) / probs[idx]
        # complex64 storage: the relative error of a probability far below 2^-n grows.
        big = probs[idx] >= 0.01 * 2.0 ** -24
        assert rel[big].max() < tol
        assert np.abs(p - probs[idx]).max() < (1e-8 if prec != "c128" else 1e-18)
    cs = pkg.ChainSampler(inst.g, inst.u, inst.order)
    sb, sp, slogp = cs.sample(1000, seed=24)
    sidx = (sb.astype(np.int64) << np.arange(24)).sum(axis=1)
    assert np.allclose(sp, probs[sidx], rtol=1e-4)
    assert np.abs(slogp - np.log(probs[sidx])).max() < 1e-4
    # Born check: linear XEB of the samples against its exact expectation 2^n sum p^2 - 1,
    # and a grouped chi-square over 32 equal-mass groups of strings.
    z = (2.0 ** 24) * probs[sidx]
    assert abs(z.mean() - (2.0 ** 24) * (probs ** 2).sum()) < 6 * z.std(ddof=1) / np.sqrt(len(z))
    G = 32
    order = np.argsort(probs, kind="stable")
    grp = np.empty(len(probs), np.int64)
    grp[order] = np.minimum((np.cumsum(probs[order]) * G).astype(np.int64), G - 1)
    e = np.bincount(grp, weights=probs, minlength=G) * len(sidx)
    c = np.bincount(grp[sidx], minlength=G)
    assert stats.chi2.sf(((c - e) ** 2 / e).sum(), G - 1) > 1e-4
