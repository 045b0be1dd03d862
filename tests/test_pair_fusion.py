"""Fused pairs of scan positions (host side, no GPU).

The compiler's pair records (``rgs_plan_pair_info``) are executed here by a NumPy
emulation of the pair kernel's group walk (groups q0 + W, A units, B units) and compared
with the two positions run one after the other by the oracle's step rule
(``scan_plan.py:161-195``): same outputs, every input row read once, every output row
written once; for RGS70 (rank 30) on sampled groups, row by row.  Also: which pairs
are chosen, and that fusion can be switched off.
"""
import numpy as np
import pytest

from oracle import scan_plan as sp

PAIR_NC = {0: 1, 1: 2, 2: 2, 3: 4, 4: 2}
PAIR_NG0 = {0: 1, 1: 1, 2: 2, 3: 2, 4: 2}


def _parity(x):
    return bin(int(x)).count("1") & 1


def _apply(cols, x):
    r = 0
    for i, c in enumerate(cols):
        if (x >> i) & 1:
            r ^= int(c)
    return r


def _oracle_step(env, st, f0, f1):
    """One free position of the oracle sweep, without renormalisation."""
    tables = sp.byte_tables(st.Lcols, st.r_out)
    out = np.zeros(1 << st.r_out, dtype=np.complex128)
    mask = (1 << st.r_in) - 1
    combos = sp.kernel_combos(st.kernel)
    for c in range(1 << st.r_out):
        p0 = 0
        for b in range(tables.shape[0]):
            p0 ^= int(tables[b][(c >> (8 * b)) & 255])
        acc = 0j
        for combo in combos:
            p = p0 ^ int(combo)
            row = p & mask
            y = (p >> st.r_in) & 1
            sign = -1.0 if (y and _parity(row & st.beta)) else 1.0
            acc += env[row] * sign * (f1 if y else f0)
        out[c] = acc
    return out


def _deposit(it, piv):
    q = it
    for p in piv:
        low = (1 << p) - 1
        q = ((q & ~low) << 1) | (q & low)
    return q


def _emulate_group(info, it, env, fa, fb):
    """The pair kernel's computation of group `it` for one item, in complex128:
    returns ([(output row, value)], [input rows read]); env(row) gives A's input."""
    ca, cb = info.code_a, info.code_b
    pair_a, pair_b = ca != 4, cb != 4
    nca, ncb = PAIR_NC[ca], PAIR_NC[cb]
    ng0a, ng0b = PAIR_NG0[ca], PAIR_NG0[cb]
    nua, nub = ncb, (2 if pair_a else 1)
    nw = 2 * ncb if pair_a else ncb
    m, dw = info.m, info.dw
    piv = [info.piv[k] for k in range(dw)]
    la = [info.la_cols[i] for i in range(m)]
    mb = [info.mb_cols[i] for i in range(m)]
    wa, wb = fa if pair_a else (fa[0] + fa[1], fa[0] - fa[1])
    va, vb = fb if pair_b else (fb[0] + fb[1], fb[0] - fb[1])
    q0 = _deposit(it, piv)
    p0 = _apply(la, q0)
    c0 = _apply(mb, q0)
    pq = _parity(q0 & info.beta_b)
    reg = [0j] * nw
    reads, outs = [], []
    for a in range(nua):
        pu = p0 ^ int(info.la_w[a])
        ya = (pu >> info.a) & 1
        terms = []
        for k in range(nca):
            row = (pu ^ int(info.comb_a[k])) & int(info.mask_a)
            reads.append(row)
            terms.append((env(row), _parity(row & info.beta_a)))
        if pair_a:
            x = y = 0j
            for k, (e, par) in enumerate(terms):
                n = -e if par else e
                if k < ng0a:
                    x += e * wa
                    y += n * wb
                else:
                    x += n * wb
                    y += e * wa
            reg[2 * a], reg[2 * a + 1] = (y, x) if ya else (x, y)
        else:
            reg[a] = sum(e * (wb if par else wa) for e, par in terms)
    for b in range(nub):
        x = y = 0j
        for a in range(ncb):
            i = (a << 1) | b if pair_a else a
            par = pq ^ ((info.pw_b >> i) & 1)
            e = reg[i]
            n = -e if par else e
            if pair_b:
                if a < ng0b:
                    x += e * va
                    y += n * vb
                else:
                    x += n * vb
                    y += e * va
            else:
                x += e * (vb if par else va)
        cx = c0 ^ int(info.mb0[b])
        outs.append((cx, x))
        if pair_b:
            outs.append((cx ^ int(info.t_b), y))
    return outs, reads


def _emulate_pair(info, env, fa, fb):
    """Every group of the pair: the full output table, write and read counts."""
    out = np.zeros(1 << info.o, dtype=np.complex128)
    written = np.zeros(1 << info.o, dtype=np.int64)
    read = np.zeros(len(env), dtype=np.int64)
    for it in range(1 << (info.m - info.dw)):
        outs, reads = _emulate_group(info, it, env.__getitem__, fa, fb)
        for row, val in outs:
            out[row] = val
            written[row] += 1
        for row in reads:
            read[row] += 1
    return out, written, read


def _oracle_at(st, c, env, f0, f1):
    """Output row c of one free position of the oracle sweep (scan_plan.py:161-195),
    without renormalisation; env(row) gives the position's input."""
    p0 = _apply(st.Lcols, c)
    mask = (1 << st.r_in) - 1
    acc = 0j
    for combo in sp.kernel_combos(st.kernel):
        p = p0 ^ int(combo)
        row = p & mask
        y = (p >> st.r_in) & 1
        sign = -1.0 if (y and _parity(row & st.beta)) else 1.0
        acc += env(row) * sign * (f1 if y else f0)
    return acc


def _instances(pkg):
    rng = np.random.default_rng(12)
    out = []
    for kind, n in (("reg3", 14), ("reg3", 18), ("er3", 16), ("deg3", 20), ("dense", 12), ("dense", 14)):
        for s in range(3):
            if kind == "dense":
                g = pkg.instances.dense(n, rng)
                order = rng.permutation(n).tolist()
                out.append((g, order))
            else:
                inst = pkg.instances.make_instance(kind, n, int(rng.integers(1 << 30)), pkg.rank_profile)
                out.append((inst.g, inst.order))
                out.append((inst.g, rng.permutation(n).tolist()))
    return out


def test_pair_records_match_two_oracle_steps(pkg):
    rng = np.random.default_rng(5)
    codes = set()
    npairs = 0
    for g, order in _instances(pkg):
        n = g.shape[0]
        edges = pkg.edges_from_graph(g)
        plan = pkg.ScanPlan(n, edges, order)
        steps, _ = sp.make_plan(n, [tuple(e) for e in edges], order)
        for k, j in enumerate(plan.pairs):
            info = plan.pair_info(k)
            assert info.j == j and 1 <= j < n - 1
            A, B = steps[j], steps[j + 1]
            if A.r_out > 12 or A.r_in > 12 or B.r_out > 12:
                continue
            env = rng.normal(size=1 << A.r_in) + 1j * rng.normal(size=1 << A.r_in)
            fa = rng.normal(size=2) + 1j * rng.normal(size=2)
            fb = rng.normal(size=2) + 1j * rng.normal(size=2)
            ref = _oracle_step(_oracle_step(env, A, *fa), B, *fb)
            got, written, read = _emulate_pair(info, env, fa, fb)
            assert np.all(written == 1), (j, info.code_a, info.code_b)
            assert np.all(read == 1), (j, info.code_a, info.code_b)
            assert np.allclose(got, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max()), (j, info.code_a, info.code_b)
            codes.add((info.code_a, info.code_b))
            npairs += 1
    assert npairs >= 40
    # Rising, peak and falling pairs of 3-regular plans, and the merge codes.
    assert {(0, 0), (0, 3), (3, 3), (3, 4), (4, 4)} <= codes, codes


def test_pairs_chosen_and_switch(pkg):
    inst = pkg.instances.make_instance("reg3", 24, 3, pkg.rank_profile)
    edges = pkg.edges_from_graph(inst.g)
    plan = pkg.ScanPlan(inst.n, edges, inst.order)
    pairs = plan.pairs
    assert pairs and all(b - a >= 2 for a, b in zip(pairs, pairs[1:]))
    assert 0 not in pairs and all(j + 1 < inst.n for j in pairs)
    # The pairs skip the largest intermediate tables: the peak rank is never materialised
    # when a pair around it is allowed.
    off = pkg.ScanPlan(inst.n, edges, inst.order, fuse=False)
    assert off.pairs == []
    # No pair straddles the low-rank head / middle / tail split of the chunked sweep
    # (positions whose input and output ranks are at most 12 run once per chunk).
    for g, order in _instances(pkg)[:12]:
        plan = pkg.ScanPlan(len(g), pkg.edges_from_graph(g), order)
        r = plan.ranks
        small = [max(r[j - 1] if j else 0, r[j]) <= 12 for j in range(len(r))]
        h = 0
        while h < len(r) and small[h]:
            h += 1
        t = len(r)
        while t > h and small[t - 1]:
            t -= 1
        region = [0 if j < h else (1 if j < t else 2) for j in range(len(r))]
        for j in plan.pairs:
            assert region[j] == region[j + 1]
    # Plans with fixed vertices are not fused.
    fx = pkg.ScanPlan(inst.n, edges, inst.order, frozenset({inst.order[3]}))
    assert fx.pairs == []


def test_fusion_switch_after_use_is_rejected(pkg):
    import ctypes
    inst = pkg.instances.make_instance("reg3", 10, 3, pkg.rank_profile)
    plan = pkg.ScanPlan(inst.n, pkg.edges_from_graph(inst.g), inst.order)
    # Before any device use the switch is accepted (host only).
    pkg._lib.check(pkg._lib.lib().rgs_plan_set_fusion(plan.handle, 0))
    pkg._lib.check(pkg._lib.lib().rgs_plan_set_fusion(plan.handle, 1))
    cnt = ctypes.c_int32()
    pkg._lib.check(pkg._lib.lib().rgs_plan_pairs(plan.handle, ctypes.byref(cnt), None))
    assert cnt.value == len(plan.pairs)


def test_rgs70_pair_records_on_sampled_groups(pkg, fixtures):
    """RGS70 (rank 30): tables are far too large to emulate whole, so sampled groups of
    every fused pair are checked output row by output row against the two oracle steps
    evaluated at that row, with table entries drawn from a seeded hash of the row."""
    g = fixtures["rgs70/graph"]
    edges = pkg.edges_from_graph(g)
    order = fixtures["rgs70/scan_order"].tolist()
    plan = pkg.ScanPlan(70, edges, order)
    steps, _ = sp.make_plan(70, [tuple(e) for e in edges], order)
    assert len(plan.pairs) >= 20

    def env(row):
        r = np.random.default_rng(int(row) * 2654435761 % (1 << 63))
        return complex(r.normal(), r.normal())

    rng = np.random.default_rng(70)
    fa = (0.6 + 0.2j, -0.3 + 0.7j)
    fb = (0.1 - 0.8j, 0.5 + 0.4j)
    for k, j in enumerate(plan.pairs):
        info = plan.pair_info(k)
        A, B = steps[j], steps[j + 1]
        for it in rng.integers(0, 1 << (info.m - info.dw), size=3):
            outs, reads = _emulate_group(info, int(it), env, fa, fb)
            assert len(set(reads)) == len(reads)
            assert len({r for r, _ in outs}) == len(outs)
            for row, val in outs:
                ref = _oracle_at(B, row, lambda q: _oracle_at(A, q, env, *fa), *fb)
                assert abs(val - ref) <= 1e-12 * max(1.0, abs(ref)), (j, row)


RARE_CODES = {(2, 2), (3, 0), (4, 0), (4, 1)}


def rare_code_plans(pkg):
    """Small seeded plans that fuse the pair codes the larger test graphs do not produce
    (a searched, deterministic list: one (graph, order) per code)."""
    found = {}
    rng = np.random.default_rng(9)
    for t in range(3000):
        n = int(rng.integers(8, 15))
        kind = t % 4
        if kind == 0:
            g = pkg.instances.dense(n, rng)
        else:
            name = ["reg3", "er3", "deg3"][kind - 1]
            if name == "reg3" and n % 2:
                name = "er3"
            g = pkg.instances.make_instance(name, n, int(rng.integers(1 << 30)), pkg.rank_profile).g
        order = rng.permutation(n).tolist()
        plan = pkg.ScanPlan(n, pkg.edges_from_graph(g), order)
        for k in range(len(plan.pairs)):
            info = plan.pair_info(k)
            c = (info.code_a, info.code_b)
            if c in RARE_CODES and c not in found:
                found[c] = (g, order)
        if len(found) == len(RARE_CODES):
            break
    return found


def test_rare_pair_codes(pkg):
    plans = rare_code_plans(pkg)
    assert set(plans) == RARE_CODES
    rng = np.random.default_rng(6)
    for code, (g, order) in plans.items():
        n = len(g)
        edges = pkg.edges_from_graph(g)
        plan = pkg.ScanPlan(n, edges, order)
        steps, _ = sp.make_plan(n, [tuple(e) for e in edges], order)
        for k, j in enumerate(plan.pairs):
            info = plan.pair_info(k)
            A, B = steps[j], steps[j + 1]
            env = rng.normal(size=1 << A.r_in) + 1j * rng.normal(size=1 << A.r_in)
            fa = rng.normal(size=2) + 1j * rng.normal(size=2)
            fb = rng.normal(size=2) + 1j * rng.normal(size=2)
            ref = _oracle_step(_oracle_step(env, A, *fa), B, *fb)
            got, written, read = _emulate_pair(info, env, fa, fb)
            assert np.all(written == 1) and np.all(read == 1), code
            assert np.allclose(got, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max()), code
