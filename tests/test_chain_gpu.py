"""GPU chain-rule sampler against the FP64 statevector oracle (complex64 tables with
float64 or float32 arithmetic, complex128 tables; the test instances have fused pairs of
positions, so the fused Gram pass runs too).

* With given uniforms the drawn strings equal the oracle's inverse-CDF draws (strings
  whose uniform lies within 1e-5 of a branch boundary are excluded: float rounding).
* Conditional marginals p(x_v = 1 | prefix) within 1e-5 (complex64) / 1e-10 (complex128).
* log p(x) from the conditionals equals log |amplitude|^2 of the sampled string.
* Philox samples follow the Born distribution (grouped chi-square, XEB).
"""
import numpy as np
import pytest
from scipy import stats

from oracle import graph_state as gs

pytestmark = pytest.mark.gpu


def _instance(pkg, kind, n, seed):
    return pkg.instances.make_instance(kind, n, seed, pkg.rank_profile)


@pytest.mark.parametrize("kind,n,seed", [("reg3", 12, 1), ("dense", 10, 2), ("er3", 14, 3), ("deg3", 16, 4)])
@pytest.mark.parametrize("precision,tol", [("c64", 1e-5), ("c64f32", 1e-4), ("c128", 1e-10)])
def test_given_uniforms_match_oracle(pkg, kind, n, seed, precision, tol):
    inst = _instance(pkg, kind, n, seed)
    probs = np.abs(gs.statevector(inst.g, inst.u)) ** 2
    cs = pkg.ChainSampler(inst.g, inst.u, inst.order, precision=precision)
    rng = np.random.default_rng(seed)
    count = 200
    uni = rng.random((count, n))
    bits, p, logp = cs.sample(count, uniforms=uni)
    matched = 0
    for i in range(count):
        ref, margins = gs.chain_sample(probs, inst.order, uni[i])
        if margins.min() < 1e-5:
            continue
        assert np.array_equal(bits[i], ref)
        idx = int((ref.astype(np.int64) << np.arange(n)).sum())
        assert abs(p[i] - probs[idx]) / probs[idx] < (1e-12 if precision == "c128" else 1e-4)
        assert abs(logp[i] - np.log(probs[idx])) < (1e-9 if precision == "c128" else 1e-4)
        matched += 1
    assert matched > 0.95 * count
    # Conditional marginals of the drawn strings (teacher forcing), equal to those met while sampling.
    cond, lp, p2 = cs.marginals(bits)
    _, _, _, cond_s = cs.sample(count, uniforms=uni, with_conditionals=True)
    assert np.abs(cond - cond_s).max() < 1e-6
    for i in range(0, count, 17):
        ref = gs.chain_conditionals(probs, inst.order, bits[i])
        assert np.abs(cond[i] - ref).max() < max(tol, 2e-7)


def test_born_distribution(pkg):
    inst = _instance(pkg, "reg3", 12, 7)
    probs = np.abs(gs.statevector(inst.g, inst.u)) ** 2
    cs = pkg.ChainSampler(inst.g, inst.u, inst.order)
    bits, p, logp = cs.sample(20000, seed=12345)
    idx = (bits.astype(np.int64) << np.arange(12)).sum(axis=1)
    assert np.allclose(p, probs[idx], rtol=1e-4)
    G = 64
    order = np.argsort(probs, kind="stable")
    cm = np.cumsum(probs[order])
    grp = np.empty(len(probs), np.int64)
    grp[order] = np.minimum((cm * G).astype(np.int64), G - 1)
    e = np.bincount(grp, weights=probs, minlength=G) * len(idx)
    c = np.bincount(grp[idx], minlength=G)
    assert stats.chi2.sf(((c - e) ** 2 / e).sum(), G - 1) > 1e-4
    z = (1 << 12) * probs[idx]
    exact = (1 << 12) * (probs ** 2).sum() - 1
    assert abs(z.mean() - 1 - exact) < 6 * z.std(ddof=1) / np.sqrt(len(z))
    # Different seeds give different samples; the same seed repeats exactly.
    b2, _, _ = cs.sample(64, seed=12345)
    b3, _, _ = cs.sample(64, seed=54321)
    assert np.array_equal(b2, bits[:64]) and not np.array_equal(b2, b3)


def test_large_instance_consistency(pkg):
    """n = 40, rank 20 (the benchmark instance family): conditionals multiply to the
    FP64 scan probability of each sample."""
    inst = pkg.instances.make_instance("reg3", 40, 40, pkg.rank_profile)
    cs = pkg.ChainSampler(inst.g, inst.u, inst.order)
    bits, p, logp = cs.sample(256, seed=9)
    so = pkg.ScanOracle(inst.g, inst.u, inst.order, fp64=True)
    p128 = so.probabilities(bits)
    assert np.max(np.abs(p - p128) / p128) < 1e-4
    assert np.max(np.abs(logp - np.log(p128))) < 1e-4
    # Born samples score far above uniform strings (linear XEB 2^n E[p] - 1 = 2^n sum p^2 - 1
    # > 0; sparse graph states are not Porter-Thomas, so it is not ~1 here).
    xeb = (2.0 ** 40) * p128.mean() - 1
    uniform = (2.0 ** 40) * so.probabilities(pkg.instances.uniform_bits(256, 40, np.random.default_rng(1))).mean() - 1
    assert xeb > 0.5 and xeb > uniform + 0.5


def test_chain_errors(pkg):
    inst = _instance(pkg, "reg3", 10, 3)
    u = inst.u.copy()
    u[2] = np.diag([1.0, 1j])  # structurally fixed vertex
    plan = pkg.ScanPlan(10, pkg.edges_from_graph(inst.g), inst.order, fixed={2})
    cs = pkg.ChainSampler(inst.g, u, inst.order, plan=plan)
    with pytest.raises(NotImplementedError):
        cs.sample(4)
    with pytest.raises(ValueError):
        pkg.ChainSampler(inst.g, inst.u, inst.order).sample(4, uniforms=np.zeros((3, 10)))


@pytest.mark.parametrize("kind,n,seed", [("reg3", 12, 1), ("deg3", 16, 4)])
def test_launch_count_matches_profiler(pkg, kind, n, seed):
    """rgs_chain_launch_count (the benchmark's gpu_launches) equals the kernels that the
    CUDA profiler sees for one sampling call: 3 batch tiles, with log p."""
    import torch
    from torch.profiler import ProfilerActivity, profile
    inst = _instance(pkg, kind, n, seed)
    cs = pkg.ChainSampler(inst.g, inst.u, inst.order, precision="c64f32", batch_tile=32)
    count = 3 * cs.batch_tile
    outs = cs._outs(count)
    cs.sample_device(count, seed=1, check=False, outs=outs)
    torch.cuda.synchronize()
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        cs.sample_device(count, seed=2, check=False, outs=outs)
        torch.cuda.synchronize()
    ours = sum(e.count for e in prof.key_averages() if "_kernel" in e.key)
    assert ours == cs.launch_count(count) == 3 * cs.launch_count(cs.batch_tile)
