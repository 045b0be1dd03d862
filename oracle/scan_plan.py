"""CPU restatement of the reference scan compiler and NumPy executor (test oracle only).

Reference: ``W/upstream_scan/scan_plan.py`` of whyihaveyou/rgs70-classical-challenge
(``W/`` = ``work/rgs_attack/``), itself adapted from dcs-rankwidth.

The scan sums a graph-state amplitude one vertex at a time.  After position j
the processed vertices only matter through their *syndrome*: for every later
vertex, the parity of its processed neighbours that were set to 1.  Syndromes
form an affine subspace ``o + span(basis)``; the environment table ``E[c]`` is
indexed by the coordinates ``c`` of a syndrome in that basis, so it holds
``2^rank`` entries.  The compiler turns a vertex order into, per position:

* ``beta``   -- which basis vectors contain the current vertex (sign parity),
* ``Lcols``  -- a right inverse of the map (c, y) -> c' onto the new basis,
* ``kernel`` -- the null space of that map (at most two vectors),

all in exact integer arithmetic.  Everything here is plain Python ints (no
width limit) so it also serves as the bit-exactness oracle for the 128-bit C++
compiler.
"""
import math

import numpy as np

__all__ = [
    "PlanStep", "future_masks", "make_plan", "byte_tables", "kernel_combos",
    "sweep", "local_vectors", "structurally_fixed", "amplitude", "rank_profile",
]


class PlanStep:
    """One compiled scan position (fields as in ``scan_plan.py:31-32``)."""

    __slots__ = ("v", "free", "r_in", "r_out", "beta", "Lcols", "kernel")

    def as_tuple(self):
        return (self.v, self.free, self.r_in, self.r_out, self.beta,
                tuple(self.Lcols), tuple(self.kernel))


def future_masks(n, edges, order):
    """Per position, the mask (over positions) of later neighbours.

    Follows ``scan_plan.py:45-55``.
    """
    where = [0] * n
    for position, vertex in enumerate(order):
        where[vertex] = position
    later = [0] * n
    for a, b in edges:
        lo, hi = sorted((where[a], where[b]))
        later[lo] |= 1 << hi
    return later


def _eliminate(vector, rows, pivot_bits):
    """Reduce ``vector`` by ``rows`` in insertion order (``scan_plan.py:35-42``).

    Returns the residual and the bitmask of rows that were added.
    """
    used = 0
    for index, (row, bit) in enumerate(zip(rows, pivot_bits)):
        if vector >> bit & 1:
            vector ^= row
            used |= 1 << index
    return vector, used


def make_plan(n, edges, order, fixed=frozenset()):
    """Compile the scan program for ``order`` (``scan_plan.py:58-105``).

    ``fixed`` lists vertices whose value y is deterministic; such positions add
    no new syndrome direction.  Returns (steps, rank profile).
    """
    later = future_masks(n, edges, order)
    basis = []
    steps, ranks = [], []
    for j in range(n):
        st = PlanStep()
        st.v = order[j]
        st.free = st.v not in fixed
        st.r_in = len(basis)
        st.beta = 0
        for i, vec in enumerate(basis):
            if vec >> j & 1:
                st.beta |= 1 << i
        # Images of the old coordinates (bit j is consumed) and of y.
        images = [vec & ~(1 << j) for vec in basis]
        if st.free:
            images.append(later[j])
        rows, pivot_bits, columns = [], [], []
        for img in images:
            residual, used = _eliminate(img, rows, pivot_bits)
            if residual:
                pivot_bits.append((residual & -residual).bit_length() - 1)
                rows.append(residual)
                used |= 1 << (len(rows) - 1)
            columns.append(used)
        st.r_out = len(rows)
        # creator[k]: the first column whose top coefficient bit is k.
        creator = {}
        for i, col in enumerate(columns):
            if col:
                top = col.bit_length() - 1
                creator.setdefault(top, i)
        right_inverse = []
        for k in range(st.r_out):
            i = creator[k]
            col = columns[i]
            pre = 1 << i
            for l in range(k):
                if col >> l & 1:
                    pre ^= right_inverse[l]
            right_inverse.append(pre)
        st.Lcols = right_inverse
        pivot_columns = set(creator.values())
        null = []
        for i, col in enumerate(columns):
            if i in pivot_columns:
                continue
            vec = 1 << i
            for k in range(st.r_out):
                if col >> k & 1:
                    vec ^= right_inverse[k]
            null.append(vec)
        st.kernel = null
        basis = rows
        steps.append(st)
        ranks.append(st.r_out)
    return steps, ranks


def rank_profile(n, edges, order, fixed=frozenset()):
    """Rank after every position (the cost model sum(2^r) uses this)."""
    return make_plan(n, edges, order, fixed)[1]


def byte_tables(cols, nbits):
    """XOR lookup tables for c -> L c, one byte of c per table (``scan_plan.py:133-145``)."""
    nbytes = max(1, (nbits + 7) // 8)
    tables = np.zeros((nbytes, 256), dtype=np.uint64)
    for b in range(nbytes):
        for value in range(256):
            acc = 0
            for t in range(8):
                i = 8 * b + t
                if i < nbits and value >> t & 1:
                    acc ^= cols[i]
            tables[b, value] = acc
    return tables


def kernel_combos(kernel):
    """All elements of span(kernel), in the reference order (``scan_plan.py:148-152``)."""
    out = [0]
    for vec in kernel:
        out = out + [c ^ vec for c in out]
    return out


def _parity_u64(x):
    x = x.copy()
    for sh in (32, 16, 8, 4, 2, 1):
        x ^= x >> np.uint64(sh)
    return x & np.uint64(1)


def sweep(steps, f, yfix, later, dtype=np.complex128):
    """Execute a compiled plan on the CPU (``scan_plan.py:161-195``).

    ``f`` maps vertex -> 2-vector, ``yfix`` maps fixed vertex -> its value.
    Returns (value, log_scale); the contraction equals value * exp(log_scale).
    The table is renormalised by its maximum modulus after every step.
    """
    env = np.ones(1, dtype=dtype)
    offset = 0
    log_scale = 0.0
    for j, st in enumerate(steps):
        f0, f1 = complex(f[st.v][0]), complex(f[st.v][1])
        ov = offset >> j & 1
        offset &= ~(1 << j)
        if not st.free:
            y = int(yfix[st.v])
            if y:
                offset ^= later[j]
        tables = byte_tables(st.Lcols, st.r_out)
        out_idx = np.arange(1 << st.r_out, dtype=np.uint64)
        p0 = np.zeros_like(out_idx)
        for b in range(tables.shape[0]):
            p0 ^= tables[b][((out_idx >> np.uint64(8 * b)) & np.uint64(255)).astype(np.int64)]
        mask = np.uint64((1 << st.r_in) - 1)
        beta = np.uint64(st.beta)
        acc = np.zeros(1 << st.r_out, dtype=dtype)
        for combo in kernel_combos(st.kernel):
            p = p0 ^ np.uint64(combo)
            c = p & mask
            sign_bit = _parity_u64(c & beta) ^ np.uint64(ov)
            gathered = env[c.astype(np.int64)]
            if st.free:
                ybit = (p >> np.uint64(st.r_in)) & np.uint64(1)
                weight = np.where(ybit == 1, f1, f0)
                negate = (ybit & sign_bit) == 1
            else:
                weight = f1 if y else f0
                negate = (np.uint64(y) & sign_bit) == 1
            acc += gathered * np.where(negate, -1.0, 1.0) * weight
        env = acc
        peak = float(np.max(np.abs(env))) if env.size else 0.0
        if peak > 0:
            env /= peak
            log_scale += math.log(peak)
    return complex(env[0]), log_scale


def local_vectors(U, n, x_bits):
    """Contraction vectors f_q = <x_q| U_q (``scan_plan.py:108-120``, data qubits only)."""
    return {q: np.asarray(U[q][int(x_bits[q])], dtype=np.complex128) for q in range(n)}


def structurally_fixed(U, n, tol=1e-12):
    """Vertices whose y is deterministic for both outcomes (``scan_plan.py:123-130``)."""
    fixed = set()
    for q in range(n):
        rows = [np.asarray(U[q][0]), np.asarray(U[q][1])]
        if all(min(abs(r[0]), abs(r[1])) < tol for r in rows):
            fixed.add(q)
    return fixed


def amplitude(g, U, order, bits, fixed=None):
    """<x| (x)U |G> for adjacency matrix ``g`` (``W/scan_oracle.py:25-29``)."""
    n = len(g)
    edges = [(i, j) for i in range(n) for j in range(i + 1, n) if g[i][j]]
    fixed = set() if fixed is None else set(fixed)
    steps, _ = make_plan(n, edges, list(order), fixed)
    f = local_vectors(U, n, bits)
    yfix = {q: (0 if abs(f[q][0]) > 1e-12 else 1) for q in fixed}
    value, log_scale = sweep(steps, f, yfix, future_masks(n, edges, list(order)))
    return value * math.exp(log_scale) * 2.0 ** (-n / 2)
