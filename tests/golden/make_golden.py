"""Generate the golden fixtures in this directory by running the REFERENCE code.

Imports whyihaveyou/rgs70-classical-challenge read-only from the checkout named by
``--reference PATH`` or the RGS_REFERENCE environment variable (there is no default)
-- it never writes there -- and stores small
input/output vectors that pin the CPU oracle (``oracle/``) and the CUDA engine:

* ``plans.json``        reference ``make_plan`` / ``future_masks`` output for
                        seeded random (graph, order, fixed) cases, and the
                        rank profile sums of the RGS70 orders;
* ``amplitudes.json``   reference ``sweep_reference`` / ``ScanOracle(gpu=False)``
                        amplitudes on seeded instances (dense, 3-regular, ER);
* ``fixtures.npz``      the reference's induced 12/24/32/40-qubit and RGS70
                        instances (graph, unitaries, A, B), the RGS70 scan
                        orders, and reference conditional / covariant /
                        deferred vectors and specialisation tables;
* ``rgs70_c128.json``   a subset of the reference's stored complex128
                        probabilities for RGS70 bitstrings (the 32-input order
                        benchmark rows and cap-1 scored records);
* ``rgs70_born.json``   the complex128 probabilities of the reference's 3,452 exact
                        Born samples of RGS70 (born/batch{1,2}/*_fp64.jsonl), the
                        empirical law of p(x) under Born sampling.

Run from the repository root:
    python tests/golden/make_golden.py --reference PATH [born]
(``born`` rewrites only rgs70_born.json).
"""
import importlib.util
import json
import os
import sys
from pathlib import Path

import numpy as np

sys.dont_write_bytecode = True

def _reference_root(argv):
    """The reference checkout: ``--reference PATH`` or $RGS_REFERENCE, else exit."""
    if "--reference" in argv:
        k = argv.index("--reference")
        if k + 1 < len(argv):
            return Path(argv[k + 1]), argv[:k] + argv[k + 2:]
    if os.environ.get("RGS_REFERENCE"):
        return Path(os.environ["RGS_REFERENCE"]), argv
    sys.exit("make_golden.py: name the reference checkout with --reference PATH or RGS_REFERENCE")


REF, ARGS = (_reference_root(sys.argv[1:]) if __name__ == "__main__" else (Path("."), []))
W = REF / "work" / "rgs_attack"
OUT = Path(__file__).resolve().parent


def load(name, path):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def random_graph(rng, n, kind):
    g = np.zeros((n, n), dtype=np.uint8)
    if kind == "dense":
        g = np.triu(rng.integers(0, 2, (n, n), dtype=np.uint8), 1)
    elif kind == "er3":
        p = min(1.0, 3.0 / max(n - 1, 1))
        g = np.triu((rng.random((n, n)) < p).astype(np.uint8), 1)
    elif kind == "reg3":
        while True:
            stubs = rng.permutation(np.repeat(np.arange(n), 3))
            pairs = stubs.reshape(-1, 2)
            ok = all(a != b for a, b in pairs) and len({tuple(sorted(p)) for p in pairs}) == len(pairs)
            if ok:
                break
        for a, b in pairs:
            g[min(a, b), max(a, b)] = 1
    g = g | g.T
    return g


def haar_su2(rng, n):
    out = []
    for _ in range(n):
        z = rng.normal(size=(2, 2)) + 1j * rng.normal(size=(2, 2))
        q, r = np.linalg.qr(z)
        q = q * (np.diag(r) / np.abs(np.diag(r)))
        q = q / np.sqrt(np.linalg.det(q))
        out.append(q)
    return np.array(out)


def edges_of(g):
    n = len(g)
    return [(i, j) for i in range(n) for j in range(i + 1, n) if g[i, j]]


def plan_record(steps, ranks, fut):
    return {
        "ranks": list(map(int, ranks)),
        "fut": [str(int(x)) for x in fut],
        "steps": [[int(s.v), bool(s.free), int(s.r_in), int(s.r_out), str(int(s.beta)),
                   [str(int(x)) for x in s.Lcols], [str(int(x)) for x in s.kernel]] for s in steps],
    }


def born_records():
    """Complex128 scores of the reference's Born samples, in file order."""
    born = REF / "born"
    out = {}
    for batch in ("batch1", "batch2"):
        probs = []
        for path in sorted((born / batch).glob("born*_group*_fp64.jsonl")):
            for line in path.read_text().splitlines():
                d = json.loads(line)
                if "probability" in d and "bitstring_q0_left" in d:
                    probs.append(d["probability"])
        out[batch] = probs
    (OUT / "rgs70_born.json").write_text(json.dumps({
        "source": "reference born/batch{1,2}/born_group*_fp64.jsonl (complex128 rescoring of its exact Born samples)",
        "n": 70, "probability_c128": out}))


def main():
    if ARGS == ["born"]:
        born_records()
        return
    born_records()
    sp = load("ref_scan_plan", W / "upstream_scan" / "scan_plan.py")
    sys.path.insert(0, str(W))
    gs = load("graph_sampler", W / "graph_sampler.py")
    fc = load("fourier_covariant_sampler", W / "fourier_covariant_sampler.py")
    dg = load("deferred_global_sampler", W / "deferred_global_sampler.py")
    ins = load("init_specialization", W / "init_specialization.py")
    so = load("scan_oracle", W / "scan_oracle.py")

    rng = np.random.default_rng(20261203)
    # ---------------------------------------------------------------- plans
    cases = []
    for idx in range(160):
        kind = ["dense", "er3", "reg3"][idx % 3]
        n = int(rng.integers(2, 13)) if idx < 60 else int(rng.integers(12, 41))
        if kind == "reg3" and n % 2:
            n += 1
        if kind == "reg3" and n < 4:
            n = 4
        g = random_graph(rng, n, kind)
        order = rng.permutation(n).tolist()
        fixed = sorted(rng.choice(n, size=int(rng.integers(0, max(1, n // 4) + 1)), replace=False).tolist()) \
            if idx % 5 == 4 else []
        edges = edges_of(g)
        steps, ranks = sp.make_plan(n, edges, order, frozenset(fixed))
        fut = sp.future_masks(n, edges, order)
        rec = {"n": n, "kind": kind, "edges": edges, "order": order, "fixed": fixed}
        rec.update(plan_record(steps, ranks, fut))
        cases.append(rec)
    rgs = np.load(W / "rgs_graph.npz")
    g70 = rgs["graph"]
    orders = {"scan_order": np.load(W / "scan_order.npy").tolist(),
              "scan_order_optimized": np.load(W / "scan_order_optimized.npy").tolist()}
    rgs_plans = {}
    for name, order in orders.items():
        steps, ranks = sp.make_plan(70, edges_of(g70), order)
        fut = sp.future_masks(70, edges_of(g70), order)
        rec = plan_record(steps, ranks, fut)
        rec["sum_states"] = int(sum(2 ** r for r in ranks))
        rec["order"] = order
        rgs_plans[name] = rec
        tables = [sp.byte_tables(s.Lcols, s.r_out) for s in steps]
        rec["tables_xor_checksum"] = str(int(np.bitwise_xor.reduce(np.concatenate([t.ravel() for t in tables]))))
        rec["combos"] = [[str(int(c)) for c in sp.kernel_combos(s.kernel)] for s in steps]
    (OUT / "plans.json").write_text(json.dumps({"cases": cases, "rgs70": rgs_plans}))

    # ---------------------------------------------------------------- amplitudes
    amps = []
    for idx in range(24):
        kind = ["dense", "er3", "reg3"][idx % 3]
        n = [6, 8, 10, 12, 14, 16, 18, 20][idx % 8]
        g = random_graph(rng, n, kind)
        u = haar_su2(rng, n)
        order = rng.permutation(n).tolist()
        edges = edges_of(g)
        steps, ranks = sp.make_plan(n, edges, order)
        fut = sp.future_masks(n, edges, order)
        full = gs.graph_vector(g)
        for q in range(n):
            gs.apply_one(full, u[q], q)
        rows = []
        for t in range(6):
            bits = rng.integers(0, 2, n).tolist()
            f = {i: u[i, bits[i], :] for i in range(n)}
            val, ls = sp.sweep_reference(steps, f, {}, fut)
            amp = val * np.exp(ls) * 2.0 ** (-n / 2)
            sv = full[sum(b << j for j, b in enumerate(bits))]
            rows.append({"bits": bits, "value": [val.real, val.imag], "logscale": ls,
                         "amplitude": [amp.real, amp.imag], "statevector": [sv.real, sv.imag]})
        amps.append({"n": n, "kind": kind, "edges": edges, "order": order,
                     "u": [[[[z.real, z.imag] for z in row] for row in m2] for m2 in u],
                     "ranks": list(map(int, ranks)), "rows": rows})
    # ScanOracle(gpu=False) on the reference's own selftest generator (W/scan_oracle.py:31-45).
    st = so.selftest(str(W / "upstream_scan"), 0, False)
    (OUT / "amplitudes.json").write_text(json.dumps({"instances": amps, "scan_oracle_cpu_selftest": st}))

    # ---------------------------------------------------------------- conditional fixtures
    arrays = {}
    for name in ("induced_12q", "induced_24q", "induced_32q", "induced_40q"):
        d = np.load(W / f"{name}.npz")
        for key in ("graph", "measurement_unitaries", "A", "B"):
            arrays[f"{name}/{key}"] = d[key]
    for key in ("graph", "measurement_unitaries", "A", "B"):
        arrays[f"rgs70/{key}"] = rgs[key]
    for name, order in orders.items():
        arrays[f"rgs70/{name}"] = np.asarray(order, dtype=np.int64)
    crng = np.random.default_rng(2026120301)
    for name in ("induced_12q", "induced_24q"):
        g = arrays[f"{name}/graph"]
        u = arrays[f"{name}/measurement_unitaries"]
        A = arrays[f"{name}/A"].tolist()
        B = arrays[f"{name}/B"].tolist()
        for t in range(3):
            ob = crng.integers(0, 2, len(B)).tolist()
            va, pb = gs.conditional(g, u, A, B, ob)
            cov = fc.cpu_covariant(g, u, A, B, ob)
            raw, final = dg.cpu_deferred(g, u, A, B, ob)
            arrays[f"{name}/cond{t}/outB"] = np.asarray(ob, dtype=np.int64)
            arrays[f"{name}/cond{t}/conditional"] = va
            arrays[f"{name}/cond{t}/marginal"] = np.float64(pb)
            arrays[f"{name}/cond{t}/covariant"] = cov
            arrays[f"{name}/cond{t}/deferred_raw"] = raw
            arrays[f"{name}/cond{t}/deferred_final"] = final
    for name in ("induced_12q", "induced_24q", "induced_32q", "induced_40q", "rgs70"):
        g = arrays[f"{name}/graph"]
        u = arrays[f"{name}/measurement_unitaries"]
        A = arrays[f"{name}/A"].tolist()
        B = arrays[f"{name}/B"].tolist()
        M = g[np.ix_(B, A)]
        arrays[f"{name}/gf2rank_BA"] = np.int64(gs.gf2rank(M))
        N = fc.gf2_inverse(M).T
        arrays[f"{name}/inverse_transpose"] = N
        ids = crng.integers(0, 1 << len(A), 4096, dtype=np.uint64)
        arrays[f"{name}/probe_ids"] = ids
        arrays[f"{name}/probe_mapped"] = fc.map_indices(ids, N)
        arrays[f"{name}/probe_phase_B"] = fc.phase_for_ids(fc.map_indices(ids, N), g[np.ix_(B, B)])
        arrays[f"{name}/probe_phase_A"] = fc.phase_for_ids(ids, g[np.ix_(A, A)])
        selected = np.asarray(u)[B]
        if np.array_equal(selected, np.broadcast_to(selected[0], selected.shape)):
            spec = ins.build_specialization(g, u, A, B)
            arrays[f"{name}/spec_tables"] = spec.packed_tables
            mx, pmask = spec.toggle_metadata(spec.m - 1)
            arrays[f"{name}/spec_toggle"] = np.array([mx, pmask], dtype=np.uint64)
            ob = crng.integers(0, 2, len(B)).tolist()
            arrays[f"{name}/spec_outB"] = np.asarray(ob, dtype=np.int64)
            arrays[f"{name}/spec_weights"] = spec.weight_table(ob, np.complex128)
            arrays[f"{name}/spec_values"] = spec.evaluate(ids, ob)
    np.savez_compressed(OUT / "fixtures.npz", **arrays)

    # ---------------------------------------------------------------- RGS70 complex128 records
    bench = json.loads((W / "cap1_full_audit_artifact" / "scan_order_benchmark.json").read_text())
    rows = [{"bitstring_q0_left": r["bitstring_q0_left"], "probability_c128": r["reference_probability"],
             "probability_c64_old": r["old_probability"], "probability_c64_new": r["new_probability"]}
            for r in bench["rows"]]
    scored = []
    for line in (W / "cap1_archive" / "scored_fp64.jsonl").read_text().splitlines():
        d = json.loads(line)
        if "bitstring_q0_left" in d:
            scored.append({"bitstring_q0_left": d["bitstring_q0_left"], "re": d["re"], "im": d["im"],
                           "probability_c128": d["probability"]})
        if len(scored) == 64:
            break
    (OUT / "rgs70_c128.json").write_text(json.dumps({
        "source": "reference complex128 reverse-order scan records",
        "benchmark_rows": rows, "scored_fp64": scored,
        "sum_states": {k: v["sum_states"] for k, v in rgs_plans.items()}}, indent=0))
    print("wrote", sorted(p.name for p in OUT.iterdir()))


if __name__ == "__main__":
    main()
