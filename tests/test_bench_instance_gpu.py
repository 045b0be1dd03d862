"""The benchmark's own instance against the oracle's NumPy sweep.

Instance: n = 40 random 3-regular graph (graph seed 40), Haar SU(2) gates, the seeded
random order with the largest max rank among 2048 seeds (r_max 20, sum 2^r 3,145,725);
the first strings of the benchmark's uniform batch (bit seed 1234).  Tolerances:
complex128 within 1e-12 relative in p(x); the float32-arithmetic complex64 bulk within
1e-4 relative for p >= 0.01 * 2^-n (the bulk's storage rounding is relative to the
table maximum, so smaller probabilities carry a larger relative error; the complex128
recheck of every result is the value a caller uses there).
"""
import numpy as np
import pytest

from oracle import scan_plan as sp

pytestmark = pytest.mark.gpu

N, GRAPH_SEED, ORDER_SEEDS, TARGET_RANK, BITS_SEED = 40, 40, range(1000, 3048), 22, 1234


def _instance(pkg):
    inst = pkg.instances.make_instance("reg3", N, GRAPH_SEED, pkg.rank_profile, target_rank=TARGET_RANK,
                                       order_seeds=ORDER_SEEDS)
    assert inst.rmax == 20 and inst.sum_states == 3145725
    return inst


def test_bench_instance_matches_oracle(pkg):
    inst = _instance(pkg)
    bits = pkg.instances.uniform_bits(65536, N, np.random.default_rng(BITS_SEED))[:8]
    ref = np.array([sp.amplitude(inst.g, inst.u, inst.order, b.tolist()) for b in bits])
    p_ref = np.abs(ref) ** 2
    assert np.all(p_ref > 0)
    p128 = pkg.ScanOracle(inst.g, inst.u, inst.order, fp64=True).probabilities(bits)
    assert np.max(np.abs(p128 - p_ref) / p_ref) < 1e-12
    for prec in ("c64f32", "c64"):
        p64 = pkg.ScanOracle(inst.g, inst.u, inst.order, precision=prec).probabilities(bits)
        big = p_ref * 2.0 ** N >= 0.01
        assert big.sum() >= 4
        assert np.max(np.abs(p64[big] - p_ref[big]) / p_ref[big]) < 1e-4
        # Below that threshold the absolute error stays at the storage rounding of the table.
        assert np.max(np.abs(p64 - p_ref)) * 2.0 ** N < 1e-4


def test_bench_instance_unfused_and_fused_agree(pkg):
    """Fused pairs (the benchmark default) and the position-by-position sweep agree."""
    inst = _instance(pkg)
    bits = pkg.instances.uniform_bits(512, N, np.random.default_rng(7))
    a = pkg.ScanOracle(inst.g, inst.u, inst.order, fp64=True).probabilities(bits)
    b = pkg.ScanOracle(inst.g, inst.u, inst.order, fp64=True, fuse=False).probabilities(bits)
    assert np.max(np.abs(a - b) / b) < 1e-12


def test_checked_probabilities_state_the_error_per_result(pkg):
    """The complex64 bulk with its error against FP64 stated per result: every returned
    probability is within 1e-4 of the complex128 scan, the stated errors are the bulk's
    own, and results whose bulk error exceeds 1e-4 come back in FP64."""
    inst = _instance(pkg)
    bits = pkg.instances.uniform_bits(4096, N, np.random.default_rng(3))
    so = pkg.ScanOracle(inst.g, inst.u, inst.order, precision="c64f32")
    p, rel, used = so.checked_probabilities(bits)
    p_bulk = so.probabilities(bits)
    p64 = pkg.ScanOracle(inst.g, inst.u, inst.order, fp64=True).probabilities(bits)
    assert np.max(np.abs(p - p64) / p64) <= 1e-4
    assert np.allclose(rel, np.abs(p_bulk - p64) / p64, rtol=1e-9, atol=0)
    assert np.array_equal(used, rel > 1e-4)
    assert np.array_equal(p[~used], p_bulk[~used]) and np.array_equal(p[used], p64[used])
    # The error is small where the probability is not far below 2^-n.
    assert rel[p64 * 2.0 ** N >= 0.01].max() < 1e-4
