"""The Gram pass of a fused pair in the chain-rule sampler (host side, no GPU).

The pair kernel's GRAM mode forms, per group, the intermediate rows of position A and,
instead of B's outputs, every output's (alpha, beta) with output = alpha f(0) + beta f(1),
accumulating G = sum (|alpha|^2, |beta|^2, alpha conj(beta)).  This NumPy emulation of
that assignment (the same group walk as the pair kernel, test_pair_fusion.py) must give
the branch masses of B: for any 2-vector f, G00 |f0|^2 + G11 |f1|^2 + 2 Re(G01 f0 conj(f1))
= the squared norm of B's output table computed by the oracle's step rule from A's output.
"""
import numpy as np

from oracle import scan_plan as sp
from test_pair_fusion import PAIR_NC, PAIR_NG0, _apply, _deposit, _instances, _oracle_step, _parity, rare_code_plans


def _gram_of_pair(info, env, fa):
    ca, cb = info.code_a, info.code_b
    pair_a, pair_b = ca != 4, cb != 4
    nca, ncb = PAIR_NC[ca], PAIR_NC[cb]
    ng0a, ng0b = PAIR_NG0[ca], PAIR_NG0[cb]
    nua, nub = ncb, (2 if pair_a else 1)
    nw = 2 * ncb if pair_a else ncb
    piv = [info.piv[k] for k in range(info.dw)]
    la = [info.la_cols[i] for i in range(info.m)]
    wa, wb = fa if pair_a else (fa[0] + fa[1], fa[0] - fa[1])
    G = np.zeros(3, dtype=np.complex128)  # G00, G11, G01
    for it in range(1 << (info.m - info.dw)):
        q0 = _deposit(it, piv)
        p0 = _apply(la, q0)
        pq = _parity(q0 & info.beta_b)
        reg = [0j] * nw
        for a in range(nua):
            pu = p0 ^ int(info.la_w[a])
            ya = (pu >> info.a) & 1
            terms = []
            for k in range(nca):
                row = (pu ^ int(info.comb_a[k])) & int(info.mask_a)
                terms.append((env[row], _parity(row & info.beta_a)))
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
            ax = bx = ay = by = 0j
            for a in range(ncb):
                i = (a << 1) | b if pair_a else a
                par = pq ^ ((info.pw_b >> i) & 1)
                e = reg[i]
                n = -e if par else e
                if pair_b:
                    if a < ng0b:
                        ax += e
                        by += n
                    else:
                        bx += n
                        ay += e
                else:
                    ax += e
                    bx += n
            pairs = [(ax, bx), (ay, by)] if pair_b else [(ax, bx)]
            for al, be in pairs:
                G += [abs(al) ** 2, abs(be) ** 2, al * np.conj(be)]
    return G


def _check(info, A, B, rng):
    env = rng.normal(size=1 << A.r_in) + 1j * rng.normal(size=1 << A.r_in)
    fa = rng.normal(size=2) + 1j * rng.normal(size=2)
    G = _gram_of_pair(info, env, fa)
    mid = _oracle_step(env, A, *fa)
    for _ in range(3):
        f = rng.normal(size=2) + 1j * rng.normal(size=2)
        mass = (G[0].real * abs(f[0]) ** 2 + G[1].real * abs(f[1]) ** 2
                + 2 * (G[2] * f[0] * np.conj(f[1])).real)
        ref = float(np.sum(np.abs(_oracle_step(mid, B, *f)) ** 2))
        assert abs(mass - ref) <= 1e-10 * ref, (info.code_a, info.code_b, mass, ref)


def test_pair_gram_gives_branch_masses(pkg):
    rng = np.random.default_rng(17)
    codes = set()
    for g, order in _instances(pkg)[:18]:
        n = g.shape[0]
        edges = pkg.edges_from_graph(g)
        plan = pkg.ScanPlan(n, edges, order)
        steps, _ = sp.make_plan(n, [tuple(e) for e in edges], order)
        for k, j in enumerate(plan.pairs):
            info = plan.pair_info(k)
            A, B = steps[j], steps[j + 1]
            if max(A.r_in, A.r_out, B.r_out) > 11:
                continue
            _check(info, A, B, rng)
            codes.add((info.code_a, info.code_b))
    assert {(0, 0), (0, 3), (3, 3), (3, 4), (4, 4)} <= codes, codes


def test_pair_gram_rare_codes(pkg):
    rng = np.random.default_rng(18)
    for code, (g, order) in rare_code_plans(pkg).items():
        n = len(g)
        edges = pkg.edges_from_graph(g)
        plan = pkg.ScanPlan(n, edges, order)
        steps, _ = sp.make_plan(n, [tuple(e) for e in edges], order)
        for k, j in enumerate(plan.pairs):
            info = plan.pair_info(k)
            _check(info, steps[j], steps[j + 1], rng)
