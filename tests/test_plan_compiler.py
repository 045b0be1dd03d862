"""The C++ scan compiler (through the C ABI, host-only) is bit-identical to the
reference's make_plan: golden cases, RGS70, and a seeded fuzz against the oracle."""
import numpy as np
import pytest

from oracle import scan_plan as sp


def _rows(steps):
    return [[s.v, s.free, s.r_in, s.r_out, str(s.beta), [str(x) for x in s.Lcols], [str(x) for x in s.kernel]]
            for s in steps]


def test_golden_cases(pkg, golden_plans):
    for case in golden_plans["cases"]:
        plan = pkg.ScanPlan(case["n"], [tuple(e) for e in case["edges"]], case["order"], frozenset(case["fixed"]))
        assert _rows(plan.steps) == case["steps"]
        assert plan.ranks == case["ranks"]
        assert [str(x) for x in plan.fut] == case["fut"]


def test_rgs70(pkg, golden_plans, fixtures):
    g = fixtures["rgs70/graph"]
    edges = pkg.edges_from_graph(g)
    for name, rec in golden_plans["rgs70"].items():
        plan = pkg.ScanPlan(70, edges, fixtures[f"rgs70/{name}"].tolist())
        assert _rows(plan.steps) == rec["steps"]
        assert plan.sum_states == rec["sum_states"]
        assert plan.rmax == 30 and plan.executable
        tabs = plan.tables
        assert str(int(np.bitwise_xor.reduce(np.concatenate([t.ravel() for t in tabs])))) == rec["tables_xor_checksum"]
        for j, st in enumerate(plan.steps[:12]):
            assert np.array_equal(tabs[j], sp.byte_tables(st.Lcols, st.r_out))
        assert [[str(c) for c in pkg.kernel_combos(s.kernel)] for s in plan.steps] == rec["combos"]


@pytest.mark.parametrize("seed", range(6))
def test_fuzz_against_oracle(pkg, seed):
    """Random graphs up to 100 vertices (masks wider than 64 bits), random orders and fixed sets."""
    rng = np.random.default_rng(1000 + seed)
    for _ in range(40):
        n = int(rng.integers(1, 101))
        p = float(rng.choice([0.05, 0.1, 0.3, 0.6]))
        g = np.triu((rng.random((n, n)) < p).astype(np.uint8), 1)
        edges = list(zip(*map(list, np.nonzero(g))))
        order = rng.permutation(n).tolist()
        fixed = frozenset(rng.choice(n, size=int(rng.integers(0, n // 3 + 1)), replace=False).tolist()) \
            if rng.random() < 0.3 else frozenset()
        plan = pkg.ScanPlan(n, edges, order, fixed)
        steps, ranks = sp.make_plan(n, edges, order, fixed)
        assert plan.ranks == ranks
        assert [s.as_tuple() for s in plan.steps] == [s.as_tuple() for s in steps]
        assert plan.fut == sp.future_masks(n, edges, order)
        assert pkg.rank_profile(n, edges, order, fixed) == ranks


def test_compiler_errors(pkg):
    with pytest.raises(ValueError):
        pkg.ScanPlan(3, [(0, 1)], [0, 1, 1])
    with pytest.raises(ValueError):
        pkg.ScanPlan(3, [(0, 3)], [0, 1, 2])
    with pytest.raises(ValueError):
        pkg.ScanPlan(2, [(1, 1)], [0, 1])
    with pytest.raises(ValueError):
        pkg.ScanPlan(129, [], list(range(129)))
    # Edge-free and single-vertex graphs compile to rank 0.
    assert pkg.ScanPlan(1, [], [0]).ranks == [0]
    assert pkg.ScanPlan(5, [], list(range(5))).rmax == 0


def test_device_modes_cover_every_step(pkg):
    """Every free step is either a pair step (y image t != 0) or a merge step."""
    rng = np.random.default_rng(5)
    for _ in range(30):
        n = int(rng.integers(2, 40))
        g = np.triu((rng.random((n, n)) < 0.2).astype(np.uint8), 1)
        edges = list(zip(*map(list, np.nonzero(g))))
        plan = pkg.ScanPlan(n, edges, rng.permutation(n).tolist())
        for st in plan.steps:
            assert len(st.kernel) <= 2
            assert st.r_out >= st.r_in - 1 and st.r_out <= st.r_in + 1


def test_chain_launch_count_host_logic(pkg):
    """rgs_chain_launch_count (the chain sampler's kernel launches, counted on the host):
    whole batch tiles, one bit-clearing kernel in sampling but not in marginals mode, one
    log p zeroing kernel when log p is asked for, and per position at most a Gram pass, a
    decision and a step (a fused pair shares the step)."""
    import ctypes
    rng = np.random.default_rng(11)
    L = pkg._lib.lib()

    def count(plan, n_items, tile, marginals, logp):
        out = ctypes.c_int64()
        pkg._lib.check(L.rgs_chain_launch_count(plan.handle, n_items, tile, marginals, logp, ctypes.byref(out)))
        return out.value

    for _ in range(10):
        n = int(rng.integers(4, 30))
        g = np.triu((rng.random((n, n)) < 0.25).astype(np.uint8), 1)
        edges = list(zip(*map(list, np.nonzero(g))))
        plan = pkg.ScanPlan(n, edges, rng.permutation(n).tolist())
        one = count(plan, 32, 32, 0, 1)
        assert count(plan, 0, 32, 0, 1) == 0
        assert count(plan, 3 * 32, 32, 0, 1) == 3 * one
        assert count(plan, 3 * 32 + 1, 32, 0, 1) == 4 * one
        assert count(plan, 32, 32, 1, 1) == one - 1
        assert count(plan, 32, 32, 0, 0) == one - 1
        assert 2 * n - len(plan.pairs) + 1 <= one - 2 <= 3 * n + 1
    with pytest.raises(ValueError):
        count(pkg.ScanPlan(4, [(0, 1)], [0, 1, 2, 3]), -1, 32, 0, 1)
