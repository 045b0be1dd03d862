"""GPU parity of the batched scan executor against the CPU oracle.

Tolerances (probability relative error): complex64 tables 1e-4 (observed ~1e-6),
complex128 tables 1e-12, against the FP64 statevector (n <= 20), the oracle's
NumPy sweep (any n), and the reference's stored complex128 RGS70 records.
"""
import numpy as np
import pytest

from conftest import graph_from_edges, unitaries_from_json
from oracle import graph_state as gs
from oracle import scan_plan as sp

pytestmark = pytest.mark.gpu

TOL = {"c64": 1e-4, "c64f32": 1e-4, "c128": 1e-12}


def prob_rel(amp, ref):
    return np.abs(np.abs(amp) ** 2 - np.abs(ref) ** 2) / np.maximum(np.abs(ref) ** 2, 1e-300)


def sv_amplitudes(g, u, bits):
    full = gs.statevector(g, u)
    idx = (np.asarray(bits, dtype=np.int64) << np.arange(len(g))).sum(axis=1)
    return full[idx]


@pytest.mark.parametrize("kind,n,seed", [("reg3", 16, 1), ("reg3", 20, 2), ("er3", 18, 3), ("dense", 12, 4),
                                         ("deg3", 19, 5)])
@pytest.mark.parametrize("precision", ["c64", "c64f32", "c128"])
def test_amplitudes_vs_statevector(pkg, kind, n, seed, precision):
    inst = pkg.instances.make_instance(kind, n, seed, pkg.rank_profile)
    rng = np.random.default_rng(seed)
    bits = pkg.instances.uniform_bits(300, n, rng)
    ref = sv_amplitudes(inst.g, inst.u, bits)
    so = pkg.ScanOracle(inst.g, inst.u, inst.order, precision=precision)
    amp = so.amplitudes(bits)
    assert prob_rel(amp, ref).max() < TOL[precision]
    if precision != "c64f32":
        assert np.abs(amp - ref).max() < (1e-6 if precision == "c64" else 1e-14) * np.abs(ref).max() * 10


def test_golden_reference_amplitudes(pkg, golden_amplitudes):
    for inst in golden_amplitudes["instances"]:
        n = inst["n"]
        g = graph_from_edges(n, inst["edges"])
        u = unitaries_from_json(inst["u"])
        bits = np.array([r["bits"] for r in inst["rows"]])
        ref = np.array([complex(*r["amplitude"]) for r in inst["rows"]])
        for fp64, tol in ((False, 1e-4), (True, 1e-12)):
            amp = pkg.ScanOracle(g, u, inst["order"], fp64=fp64).amplitudes(bits)
            assert prob_rel(amp, ref).max() < tol


@pytest.mark.parametrize("precision", ["c64", "c64f32", "c128"])
def test_batch_tile_invariance(pkg, precision):
    """Each item's arithmetic does not depend on the batch tile: results are bitwise equal."""
    inst = pkg.instances.make_instance("reg3", 22, 9, pkg.rank_profile)
    bits = pkg.instances.uniform_bits(300, 22, np.random.default_rng(9))
    outs = []
    for tile in (1, 2, 4, 16, 32, 64, 128):
        eng = pkg.ScanEngine(pkg.ScanPlan(22, pkg.edges_from_graph(inst.g), inst.order), inst.u,
                             precision=precision, batch_tile=tile)
        outs.append(eng.sweep_bits(bits))
    for val, ls in outs[1:]:
        assert np.array_equal(val, outs[0][0]) and np.array_equal(ls, outs[0][1])


def test_contraction_vector_interface(pkg):
    """GPUMixin._sweep(f, yfix) contract with arbitrary bra vectors, against the oracle sweep."""
    inst = pkg.instances.make_instance("er3", 24, 13, pkg.rank_profile)
    n = inst.n
    rng = np.random.default_rng(13)
    edges = pkg.edges_from_graph(inst.g)
    steps, _ = sp.make_plan(n, edges, inst.order)
    fut = sp.future_masks(n, edges, inst.order)
    so = pkg.ScanOracle(inst.g, inst.u, inst.order, fp64=True)
    for _ in range(4):
        f = {q: rng.normal(size=2) + 1j * rng.normal(size=2) for q in range(n)}
        val, ls = so.engine._sweep(f, {})
        rv, rls = sp.sweep(steps, f, {}, fut)
        got, ref = val * np.exp(ls), rv * np.exp(rls)
        assert abs(got - ref) <= 1e-12 * abs(ref)
    # Bits interface == contraction-vector interface with rows of U.
    bits = pkg.instances.uniform_bits(16, n, rng)
    fvec = np.stack([inst.u[np.arange(n), b, :] for b in bits])
    v1, l1 = so.engine.sweep_bits(bits)
    v2, l2 = so.engine.sweep_fvec(fvec)
    assert np.array_equal(v1, v2) and np.array_equal(l1, l2)


def test_fixed_vertices(pkg):
    """Plans with structurally fixed vertices (diagonal / anti-diagonal U) and affine offsets."""
    rng = np.random.default_rng(21)
    for trial in range(4):
        n = 14
        g = pkg.instances.regular3(n, rng) if trial % 2 == 0 else pkg.instances.dense(n, rng)
        u = pkg.instances.haar_su2(n, rng)
        fixed_q = rng.choice(n, size=5, replace=False)
        for k, q in enumerate(fixed_q):
            ph = np.exp(1j * rng.uniform(0, 2 * np.pi, 2))
            u[q] = np.diag(ph) if k % 2 == 0 else np.array([[0, ph[0]], [ph[1], 0]])
        fixed = sp.structurally_fixed(u, n)
        assert set(fixed) == set(fixed_q.tolist())
        order = rng.permutation(n).tolist()
        edges = pkg.edges_from_graph(g)
        plan = pkg.ScanPlan(n, edges, order, fixed)
        bits = pkg.instances.uniform_bits(64, n, rng)
        ref = sv_amplitudes(g, u, bits)
        for prec, tol in (("c64", 1e-4), ("c128", 1e-12)):
            eng = pkg.ScanEngine(plan, u, precision=prec)
            val, ls = eng.sweep_bits(bits)
            amp = pkg.amplitudes_from(val, ls, n)
            mask = np.abs(ref) > 1e-12
            assert np.all(np.abs(amp[~mask]) < 1e-12)
            assert prob_rel(amp[mask], ref[mask]).max() < tol


def test_wide_instance_beyond_64_qubits(pkg):
    """n = 100 (bitstring words above 64 bits) against the oracle's NumPy sweep."""
    rng = np.random.default_rng(31)
    n = 100
    g = pkg.instances.degree_at_most3(n, rng, edge_fraction=0.6)
    u = pkg.instances.haar_su2(n, rng)
    # A breadth-first order keeps the rank small enough for the CPU oracle.
    order, seen = [], set()
    for s in range(n):
        if s in seen:
            continue
        queue = [s]
        seen.add(s)
        while queue:
            a = queue.pop(0)
            order.append(a)
            for b in np.flatnonzero(g[a]):
                if b not in seen:
                    seen.add(int(b))
                    queue.append(int(b))
    so = pkg.ScanOracle(g, u, order, fp64=True)
    assert so.rmax <= 14
    bits = pkg.instances.uniform_bits(6, n, rng)
    amp = so.amplitudes(bits)
    for b, a in zip(bits, amp):
        ref = sp.amplitude(g, u, order, b)
        assert abs(a - ref) <= 1e-12 * abs(ref)


def test_edge_cases(pkg):
    # Single vertex, edge-free graphs (product states), isolated vertices.
    for n, edges in ((1, []), (5, []), (6, [(0, 1), (2, 3)])):
        g = graph_from_edges(n, edges)
        u = pkg.instances.haar_su2(n, np.random.default_rng(n))
        bits = (np.arange(1 << n)[:, None] >> np.arange(n)) & 1
        ref = sv_amplitudes(g, u, bits)
        for fp64, tol in ((False, 1e-4), (True, 1e-12)):
            amp = pkg.ScanOracle(g, u, list(range(n))[::-1], fp64=fp64).amplitudes(bits)
            assert prob_rel(amp, ref).max() < tol
    g = graph_from_edges(4, [(0, 1), (1, 2), (2, 3)])
    so = pkg.ScanOracle(g, pkg.instances.haar_su2(4, np.random.default_rng(0)), [0, 1, 2, 3])
    with pytest.raises(ValueError):
        so.amplitudes(np.zeros((2, 5), dtype=np.uint8))
    with pytest.raises(ValueError):
        so.amplitudes(np.full((2, 4), 2, dtype=np.uint8))
    assert so.engine.sweep_bits(np.zeros((0, 4), dtype=np.uint8))[0].shape == (0,)
    with pytest.raises(ValueError):
        pkg.ScanOracle(g, so.u, [0, 1, 2, 3], gpu=False)


@pytest.mark.parametrize("fp64", [False, True])
def test_rgs70_reference_records(pkg, fixtures, rgs70_records, fp64):
    """RGS70 (n = 70, rank 30, frozen order) against the reference's complex128 records."""
    g = fixtures["rgs70/graph"]
    u = fixtures["rgs70/measurement_unitaries"]
    order = fixtures["rgs70/scan_order"].tolist()
    so = pkg.ScanOracle(g, u, order, fp64=fp64)
    rows = rgs70_records["benchmark_rows"][:4] + rgs70_records["scored_fp64"][:2]
    bits = np.array([[int(c) for c in r["bitstring_q0_left"]] for r in rows])
    p = so.probabilities(bits)
    ref = np.array([r["probability_c128"] for r in rows])
    rel = np.abs(p - ref) / ref
    assert rel.max() < (1e-12 if fp64 else 1e-4), rel


def test_autotuned_tile(pkg):
    """batch_tile='tune' measures the candidate tiles on this GPU and keeps the fastest;
    the result does not depend on the tile (bitwise)."""
    inst = pkg.instances.make_instance("reg3", 22, 9, pkg.rank_profile)
    plan = pkg.ScanPlan(22, pkg.edges_from_graph(inst.g), inst.order)
    bits = pkg.instances.uniform_bits(300, 22, np.random.default_rng(3))
    for prec in ("c64f32", "c128"):
        tuned = pkg.ScanEngine(plan, inst.u, precision=prec, batch_tile="tune")
        val, ls = tuned.sweep_bits(bits)
        best, rates = tuned.tuning
        assert tuned.batch_tile == best and best in rates and rates[best] == max(rates.values())
        ref = pkg.ScanEngine(plan, inst.u, precision=prec, batch_tile=8).sweep_bits(bits)
        assert np.array_equal(val, ref[0]) and np.array_equal(ls, ref[1])
