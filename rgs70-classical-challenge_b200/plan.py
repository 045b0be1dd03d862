"""Scan-program compiler, Python face of ``rgs_plan_*`` (C++ in ``csrc/plan.cpp``).

Mirrors ``W/upstream_scan/scan_plan.py`` of whyihaveyou/rgs70-classical-challenge
(``W/`` = ``work/rgs_attack/``): ``make_plan``, ``future_masks``, ``byte_tables``,
``kernel_combos`` and the ``Step`` record, with the same argument meanings and
bit-identical results.  Masks are Python ints (they can exceed 64 bits: n <= 128).
"""
import ctypes

import numpy as np

from . import _lib

__all__ = ["Step", "ScanPlan", "make_plan", "future_masks", "rank_profile", "search_order", "byte_tables", "kernel_combos",
           "edges_from_graph"]


class Step:
    """One compiled scan position (``scan_plan.py:31-32``)."""

    __slots__ = ("v", "free", "r_in", "r_out", "beta", "Lcols", "kernel")

    def as_tuple(self):
        return (self.v, self.free, self.r_in, self.r_out, self.beta, tuple(self.Lcols), tuple(self.kernel))

    def __repr__(self):
        return f"Step(v={self.v}, free={self.free}, r_in={self.r_in}, r_out={self.r_out})"


def edges_from_graph(g):
    """Upper-triangle edge list of a 0/1 adjacency matrix (``W/scan_oracle.py:15``)."""
    g = np.asarray(g)
    iu, ju = np.nonzero(np.triu(g, 1))
    return list(zip(iu.tolist(), ju.tolist()))


def _graph_args(n, edges, order, fixed):
    e = np.ascontiguousarray(np.asarray(list(edges), dtype=np.int32).reshape(-1, 2))
    o = np.ascontiguousarray(np.asarray(list(order), dtype=np.int32))
    if o.shape != (n,):
        raise ValueError("order must have n entries")
    f = None
    if fixed:
        f = np.zeros(n, dtype=np.uint8)
        for q in fixed:
            f[int(q)] = 1
    return e, o, f


def _u128(lo, hi):
    return int(lo) | (int(hi) << 64)


class ScanPlan:
    """A compiled scan order (opaque native handle plus exported views)."""

    def __init__(self, n, edges, order, fixed=frozenset(), fuse=True):
        L = _lib.lib()
        self.n = int(n)
        self.edges = [tuple(map(int, x)) for x in edges]
        self.order = [int(x) for x in order]
        self.fixed = frozenset(int(x) for x in fixed)
        e, o, f = _graph_args(self.n, self.edges, self.order, self.fixed)
        handle = ctypes.c_void_p()
        _lib.check(L.rgs_plan_compile(self.n, len(e), _lib.ptr(e, ctypes.c_int32), _lib.ptr(o, ctypes.c_int32),
                                      None if f is None else _lib.ptr(f, ctypes.c_uint8), ctypes.byref(handle)))
        self._h = handle
        if not fuse:
            _lib.check(L.rgs_plan_set_fusion(self._h, 0))
        n32, rmax, ex = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        _lib.check(L.rgs_plan_info(self._h, ctypes.byref(n32), ctypes.byref(rmax), ctypes.byref(ex)))
        self.rmax = int(rmax.value)
        self.executable = bool(ex.value)
        r = np.zeros(self.n, dtype=np.int32)
        _lib.check(L.rgs_plan_ranks(self._h, _lib.ptr(r, ctypes.c_int32)))
        self.ranks = r.tolist()
        self._steps = None

    @property
    def handle(self):
        return self._h

    @property
    def pairs(self):
        """Positions j whose pair (j, j + 1) runs fused (one pass, no intermediate table)."""
        L = _lib.lib()
        cnt = ctypes.c_int32()
        _lib.check(L.rgs_plan_pairs(self._h, ctypes.byref(cnt), None))
        out = np.zeros(max(1, cnt.value), dtype=np.int32)
        _lib.check(L.rgs_plan_pairs(self._h, ctypes.byref(cnt), _lib.ptr(out, ctypes.c_int32)))
        return out[:cnt.value].tolist()

    def pair_info(self, k):
        """The k-th fused pair's record (``rgs_pair_info``)."""
        info = _lib.PairInfo()
        _lib.check(_lib.lib().rgs_plan_pair_info(self._h, int(k), ctypes.byref(info)))
        return info

    @property
    def sum_states(self):
        """Cost model sum_j 2^{r_j} (``search_summary.json`` baseline_cost)."""
        return int(sum(1 << r for r in self.ranks))

    @property
    def fut(self):
        out = np.zeros(2 * self.n, dtype=np.uint64)
        _lib.check(_lib.lib().rgs_plan_future_masks(self._h, _lib.ptr(out, ctypes.c_uint64)))
        return [_u128(out[2 * j], out[2 * j + 1]) for j in range(self.n)]

    @property
    def steps(self):
        if self._steps is None:
            L = _lib.lib()
            steps = []
            for j in range(self.n):
                v, fr, ri, ro, nk = (ctypes.c_int32() for _ in range(5))
                beta = np.zeros(2, dtype=np.uint64)
                lcols = np.zeros(2 * max(1, self.ranks[j]), dtype=np.uint64)
                kern = np.zeros(4, dtype=np.uint64)
                _lib.check(L.rgs_plan_step(self._h, j, ctypes.byref(v), ctypes.byref(fr), ctypes.byref(ri),
                                           ctypes.byref(ro), _lib.ptr(beta, ctypes.c_uint64),
                                           _lib.ptr(lcols, ctypes.c_uint64), ctypes.byref(nk),
                                           _lib.ptr(kern, ctypes.c_uint64)))
                st = Step()
                st.v, st.free, st.r_in, st.r_out = v.value, bool(fr.value), ri.value, ro.value
                st.beta = _u128(beta[0], beta[1])
                st.Lcols = [_u128(lcols[2 * k], lcols[2 * k + 1]) for k in range(st.r_out)]
                st.kernel = [_u128(kern[2 * k], kern[2 * k + 1]) for k in range(nk.value)]
                steps.append(st)
            self._steps = steps
        return self._steps

    def step_tables(self, j):
        """Byte tables of step j as uint64 [nbytes, 256] (``scan_plan.py:133-145``)."""
        L = _lib.lib()
        nb = ctypes.c_int32()
        _lib.check(L.rgs_plan_step_tables(self._h, j, None, ctypes.byref(nb)))
        raw = np.zeros(nb.value * 256 * 2, dtype=np.uint64)
        _lib.check(L.rgs_plan_step_tables(self._h, j, _lib.ptr(raw, ctypes.c_uint64), ctypes.byref(nb)))
        raw = raw.reshape(nb.value, 256, 2)
        if np.any(raw[:, :, 1]):
            raise ValueError("table entries exceed 64 bits")
        return np.ascontiguousarray(raw[:, :, 0])

    @property
    def tables(self):
        return [self.step_tables(j) for j in range(self.n)]

    @property
    def combos(self):
        return [np.array(kernel_combos(st.kernel), dtype=np.uint64) for st in self.steps]

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.lib().rgs_plan_destroy(h)
            except Exception:
                pass
            self._h = None


def make_plan(N, edges, order, fixed=frozenset()):
    """(steps, rank profile), as ``scan_plan.make_plan`` (``scan_plan.py:58-105``)."""
    p = ScanPlan(N, edges, order, fixed)
    return p.steps, p.ranks


def future_masks(N, edges, order):
    """Later-neighbour masks per position (``scan_plan.py:45-55``)."""
    return ScanPlan(N, edges, order).fut


def rank_profile(N, edges, order, fixed=frozenset()):
    """Rank profile only, without keeping a plan."""
    e, o, f = _graph_args(int(N), edges, order, fixed)
    r = np.zeros(int(N), dtype=np.int32)
    _lib.check(_lib.lib().rgs_rank_profile(int(N), len(e), _lib.ptr(e, ctypes.c_int32), _lib.ptr(o, ctypes.c_int32),
                                           None if f is None else _lib.ptr(f, ctypes.c_uint8),
                                           _lib.ptr(r, ctypes.c_int32)))
    return r.tolist()


def search_order(N, edges, order, max_rank=None, iterations=100000, seed=0, threads=1):
    """Scan-order search (``W/order_optimization/search.cpp``): annealed order minimising
    sum_j 2^{r_j} with max r_j <= max_rank (default: the starting order's peak).
    Returns (order, ranks, cost)."""
    e, o, _ = _graph_args(int(N), edges, order, frozenset())
    out = np.zeros(int(N), dtype=np.int32)
    ranks = np.zeros(int(N), dtype=np.int32)
    cost = ctypes.c_double()
    _lib.check(_lib.lib().rgs_order_search(int(N), len(e), _lib.ptr(e, ctypes.c_int32), _lib.ptr(o, ctypes.c_int32),
                                           -1 if max_rank is None else int(max_rank), int(iterations),
                                           int(seed) & (2 ** 64 - 1), int(threads), _lib.ptr(out, ctypes.c_int32),
                                           _lib.ptr(ranks, ctypes.c_int32), ctypes.byref(cost)))
    return out.tolist(), ranks.tolist(), float(cost.value)


def byte_tables(cols, nbits):
    """XOR lookup tables c -> L c, one byte of c per table (``scan_plan.py:133-145``)."""
    nb = max(1, (nbits + 7) // 8)
    T = np.zeros((nb, 256), dtype=np.uint64)
    vals = np.arange(256)
    for b in range(nb):
        acc = np.zeros(256, dtype=object)
        for t in range(8):
            i = 8 * b + t
            if i < nbits:
                acc = np.where((vals >> t) & 1, acc ^ int(cols[i]), acc)
        T[b] = np.array([int(x) for x in acc], dtype=np.uint64)
    return T


def kernel_combos(kernel):
    """span(kernel) in doubling order (``scan_plan.py:148-152``)."""
    out = [0]
    for k in kernel:
        out = out + [c ^ int(k) for c in out]
    return out
