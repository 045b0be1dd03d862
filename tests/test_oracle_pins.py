"""Pin the CPU oracle to the reference: golden vectors produced by running the
reference code (tests/golden/make_golden.py) and the reference's stored records."""
import numpy as np
import pytest

from conftest import graph_from_edges, unitaries_from_json
from oracle import graph_state as gs
from oracle import scan_plan as sp


def _plan_rows(steps):
    return [[s.v, s.free, s.r_in, s.r_out, str(s.beta), [str(x) for x in s.Lcols], [str(x) for x in s.kernel]]
            for s in steps]


def test_make_plan_matches_reference(golden_plans):
    for case in golden_plans["cases"]:
        edges = [tuple(e) for e in case["edges"]]
        steps, ranks = sp.make_plan(case["n"], edges, case["order"], frozenset(case["fixed"]))
        assert _plan_rows(steps) == case["steps"]
        assert ranks == case["ranks"]
        assert [str(x) for x in sp.future_masks(case["n"], edges, case["order"])] == case["fut"]


def test_rgs70_plans_and_cost(golden_plans, fixtures, rgs70_records):
    g = fixtures["rgs70/graph"]
    edges = [(i, j) for i in range(70) for j in range(i + 1, 70) if g[i, j]]
    assert len(edges) == 1150
    for name, rec in golden_plans["rgs70"].items():
        order = fixtures[f"rgs70/{name}"].tolist()
        steps, ranks = sp.make_plan(70, edges, order)
        assert _plan_rows(steps) == rec["steps"]
        assert sum(2 ** r for r in ranks) == rec["sum_states"] == rgs70_records["sum_states"][name]
        assert max(ranks) == 30
        tabs = [sp.byte_tables(s.Lcols, s.r_out) for s in steps]
        assert str(int(np.bitwise_xor.reduce(np.concatenate([t.ravel() for t in tabs])))) == rec["tables_xor_checksum"]
        assert [[str(c) for c in sp.kernel_combos(s.kernel)] for s in steps] == rec["combos"]
    # Published cost figures (W/order_optimization/search_summary.json).
    assert rgs70_records["sum_states"]["scan_order"] == 9982443517
    assert rgs70_records["sum_states"]["scan_order_optimized"] == 7919632381


def test_sweep_matches_reference_and_statevector(golden_amplitudes):
    worst = 0.0
    for inst in golden_amplitudes["instances"]:
        n = inst["n"]
        g = graph_from_edges(n, inst["edges"])
        u = unitaries_from_json(inst["u"])
        full = gs.statevector(g, u)
        for row in inst["rows"]:
            amp = sp.amplitude(g, u, inst["order"], row["bits"])
            ref = complex(*row["amplitude"])
            idx = sum(b << j for j, b in enumerate(row["bits"]))
            assert abs(full[idx] - complex(*row["statevector"])) < 1e-15
            worst = max(worst, abs(amp - ref) / abs(ref))
    assert worst < 1e-12


def test_statevector_matches_reference_selftest(golden_amplitudes):
    st = golden_amplitudes["scan_oracle_cpu_selftest"]
    assert st["backend"] == "cpu" and st["worst_probability_relative_error"] < 1e-12
    # Re-run the reference selftest generator (W/scan_oracle.py:31-45) with the oracle.
    rng = np.random.default_rng(20261030)
    k = 0
    for n in [8, 10, 12]:
        g = rng.integers(0, 2, (n, n), dtype=np.uint8)
        g = np.triu(g, 1)
        g ^= g.T
        u = []
        for _ in range(n):
            q, _r = np.linalg.qr(rng.normal(size=(2, 2)) + 1j * rng.normal(size=(2, 2)))
            u.append(q)
        u = np.array(u)
        v = gs.statevector(g, u)
        order = rng.permutation(n).tolist()
        for _ in range(5):
            bits = rng.integers(0, 2, n).tolist()
            amp = sp.amplitude(g, u, order, bits)
            ref = v[sum(b << j for j, b in enumerate(bits))]
            assert abs(amp - ref) < 1e-12
            rel = abs(abs(amp) ** 2 - abs(ref) ** 2) / max(abs(ref) ** 2, 1e-30)
            assert abs(rel - st["cases"][k]["probability_relative_error"]) < 1e-9
            k += 1


@pytest.mark.parametrize("name", ["induced_12q", "induced_24q"])
def test_conditional_family_matches_reference(fixtures, name):
    g = fixtures[f"{name}/graph"]
    u = fixtures[f"{name}/measurement_unitaries"]
    A = fixtures[f"{name}/A"].tolist()
    B = fixtures[f"{name}/B"].tolist()
    for t in range(3):
        ob = fixtures[f"{name}/cond{t}/outB"].tolist()
        va, pb = gs.conditional(g, u, A, B, ob)
        assert np.allclose(va, fixtures[f"{name}/cond{t}/conditional"], atol=1e-14)
        assert abs(pb - float(fixtures[f"{name}/cond{t}/marginal"])) < 1e-14
        cov = gs.cpu_covariant(g, u, A, B, ob)
        assert np.allclose(cov, fixtures[f"{name}/cond{t}/covariant"], atol=1e-13)
        raw, final = gs.cpu_deferred(g, u, A, B, ob)
        assert np.allclose(raw, fixtures[f"{name}/cond{t}/deferred_raw"], atol=1e-13)
        assert np.allclose(final, fixtures[f"{name}/cond{t}/deferred_final"], atol=1e-13)
        # Full-rank cut: x_B is uniform (graph_sampler.py:158) and the covariant state is normalised.
        assert abs(pb - 2.0 ** (-len(B))) < 1e-12
        assert np.allclose(cov, va / np.sqrt(pb), atol=1e-12)


@pytest.mark.parametrize("name", ["induced_12q", "induced_24q", "induced_32q", "induced_40q", "rgs70"])
def test_gf2_maps_and_phases_bit_exact(fixtures, name):
    g = fixtures[f"{name}/graph"]
    A = fixtures[f"{name}/A"].tolist()
    B = fixtures[f"{name}/B"].tolist()
    M = g[np.ix_(B, A)]
    assert gs.gf2rank(M) == int(fixtures[f"{name}/gf2rank_BA"]) == len(A)
    N = gs.gf2_inverse(M).T
    assert np.array_equal(N, fixtures[f"{name}/inverse_transpose"])
    ids = fixtures[f"{name}/probe_ids"]
    assert np.array_equal(gs.map_indices(ids, N), fixtures[f"{name}/probe_mapped"])
    assert np.array_equal(gs.phase_for_ids(gs.map_indices(ids, N), g[np.ix_(B, B)]), fixtures[f"{name}/probe_phase_B"])
    assert np.array_equal(gs.phase_for_ids(ids, g[np.ix_(A, A)]), fixtures[f"{name}/probe_phase_A"])
    if f"{name}/spec_tables" in fixtures:
        lut, _N, _Q, _lin = gs.specialization_tables(g, A, B)
        assert np.array_equal(lut, fixtures[f"{name}/spec_tables"])
        b, phase = gs.specialization_map_and_phase(lut, ids)
        assert np.array_equal(b, fixtures[f"{name}/probe_mapped"])
        assert np.array_equal(phase, fixtures[f"{name}/probe_phase_B"])
        u = fixtures[f"{name}/measurement_unitaries"]
        ob = fixtures[f"{name}/spec_outB"].tolist()
        w = gs.specialization_weight_table(u[B[0]], ob, len(B))
        assert np.allclose(w, fixtures[f"{name}/spec_weights"], rtol=1e-14, atol=0)
        vals = w[gs.popcount64(b), gs.popcount64(b & np.uint64(sum(int(x) << j for j, x in enumerate(ob))))] * phase
        assert np.allclose(vals, fixtures[f"{name}/spec_values"], rtol=1e-13, atol=0)


def test_rgs70_born_fixture_matches_published_xeb():
    """The reference's Born-sample scores reproduce its published linear XEB
    (born/README.md: 1.096 +- 0.035, 0.953 +- 0.033, pooled 1.025 +- 0.024)."""
    import json
    from conftest import GOLDEN
    d = json.loads((GOLDEN / "rgs70_born.json").read_text())["probability_c128"]
    z1 = np.array(d["batch1"]) * 2.0 ** 70
    z2 = np.array(d["batch2"]) * 2.0 ** 70
    assert len(z1) == len(z2) == 1726
    assert abs(z1.mean() - 1 - 1.096) < 5e-4 and abs(z1.std(ddof=1) / np.sqrt(1726) - 0.035) < 5e-4
    assert abs(z2.mean() - 1 - 0.953) < 5e-4 and abs(z2.std(ddof=1) / np.sqrt(1726) - 0.033) < 5e-4
    zz = np.concatenate([z1, z2])
    assert abs(zz.mean() - 1 - 1.025) < 5e-4 and abs(zz.std(ddof=1) / np.sqrt(len(zz)) - 0.024) < 5e-4
