"""CPU statevector and conditional-state oracles (test oracle only).

Restates, from whyihaveyou/rgs70-classical-challenge (``W/`` = ``work/rgs_attack/``):

* ``W/graph_sampler.py:59-109``              gf2rank, apply_one, quadratic_phase,
                                              graph_vector, walsh, conditional
* ``W/fourier_covariant_sampler.py:23-74``   gf2_inverse, row_masks, parity64,
                                              map_indices, phase_for_ids, cpu_covariant
* ``W/deferred_global_sampler.py:93-107``    cpu_deferred
* ``W/init_specialization.py:38-189``        popcount64, transformed_quadratic,
                                              specialization lookup tables

Conventions (``W/graph_sampler.py:1``): qubit 0 is the least significant bit
of a statevector index.  All arithmetic is complex128 / exact integers.
"""
import math

import numpy as np

HADAMARD = np.array([[1, 1], [1, -1]], dtype=np.complex128)


# ----------------------------------------------------------------------------- GF(2) helpers
def gf2rank(a):
    """Rank over GF(2) of a 0/1 matrix (``graph_sampler.py:59-69``)."""
    a = np.array(a, dtype=np.uint8) & 1
    rank = 0
    rows, cols = a.shape
    for c in range(cols):
        if rank == rows:
            break
        hits = np.flatnonzero(a[rank:, c])
        if not len(hits):
            continue
        p = rank + int(hits[0])
        a[[rank, p]] = a[[p, rank]]
        below = np.flatnonzero(a[rank + 1:, c]) + rank + 1
        a[below] ^= a[rank]
        rank += 1
    return rank


def gf2_inverse(matrix):
    """Inverse of a square 0/1 matrix over GF(2) (``fourier_covariant_sampler.py:23-36``)."""
    m = np.asarray(matrix, dtype=np.uint8) & 1
    n = m.shape[0]
    if m.shape != (n, n):
        raise ValueError("square matrix required")
    aug = np.concatenate([m.copy(), np.eye(n, dtype=np.uint8)], axis=1)
    for col in range(n):
        hits = np.flatnonzero(aug[col:, col])
        if not len(hits):
            raise ValueError("singular GF(2) matrix")
        p = col + int(hits[0])
        aug[[col, p]] = aug[[p, col]]
        others = [r for r in np.flatnonzero(aug[:, col]) if r != col]
        aug[others] ^= aug[col]
    inv = aug[:, n:].copy()
    assert np.array_equal((m.astype(np.int64) @ inv) & 1, np.eye(n, dtype=np.int64))
    return inv


def row_masks(matrix):
    """Row i of a 0/1 matrix as an integer bitmask over columns."""
    return np.asarray([sum(1 << int(j) for j in np.flatnonzero(row)) for row in np.asarray(matrix)],
                      dtype=np.uint64)


def parity64(values):
    """Parity of each uint64 (``fourier_covariant_sampler.py:43-46``)."""
    y = np.asarray(values, dtype=np.uint64).copy()
    for sh in (32, 16, 8, 4, 2, 1):
        y ^= y >> np.uint64(sh)
    return y & np.uint64(1)


def popcount64(values):
    """Population count of each uint64 (``init_specialization.py:38-43``)."""
    x = np.asarray(values, dtype=np.uint64)
    out = np.zeros(x.shape, dtype=np.int64)
    for sh in range(64):
        out += ((x >> np.uint64(sh)) & np.uint64(1)).astype(np.int64)
    return out


def map_indices(ids, matrix):
    """GF(2) matrix-vector product on index bits: bit j of the result is row_j . id
    (``fourier_covariant_sampler.py:49-53``)."""
    ids = np.asarray(ids, dtype=np.uint64)
    out = np.zeros_like(ids)
    for j, mask in enumerate(row_masks(matrix)):
        out |= parity64(ids & mask) << np.uint64(j)
    return out


def upper_masks(g):
    """Row i of the strict upper triangle of ``g`` as a bitmask (``distributed_sampler.py:57``)."""
    g = np.asarray(g)
    return np.array([sum(1 << int(j) for j in np.flatnonzero(g[i, i + 1:]) + i + 1) for i in range(len(g))],
                    dtype=np.uint64)


def phase_for_ids(ids, graph):
    """(-1)^{q(b)} with q(b) = sum_{i<j} g_ij b_i b_j (``fourier_covariant_sampler.py:56-61``)."""
    ids = np.asarray(ids, dtype=np.uint64)
    par = np.zeros_like(ids)
    for i, mask in enumerate(upper_masks(graph)):
        par ^= ((ids >> np.uint64(i)) & np.uint64(1)) * parity64(ids & mask)
    return 1.0 - 2.0 * par.astype(np.float64)


# ----------------------------------------------------------------------------- statevectors
def apply_one(v, u, q):
    """Apply the 2x2 matrix u to qubit q of v in place (``graph_sampler.py:71-74``)."""
    view = v.reshape(-1, 2, 1 << q)
    a = view[:, 0, :].copy()
    b = view[:, 1, :].copy()
    view[:, 0, :] = u[0, 0] * a + u[0, 1] * b
    view[:, 1, :] = u[1, 0] * a + u[1, 1] * b


def quadratic_phase(v, g):
    """Multiply v[x] by (-1)^{sum_{a<b} g_ab x_a x_b} in place (``graph_sampler.py:76-85``)."""
    v *= phase_for_ids(np.arange(len(v), dtype=np.uint64), g)


def graph_vector(g):
    """|G> = 2^{-n/2} sum_y (-1)^{y^T Q y} |y> (``graph_sampler.py:87-88``)."""
    n = len(g)
    v = np.full(1 << n, 2.0 ** (-n / 2), dtype=np.complex128)
    quadratic_phase(v, g)
    return v


def walsh(v):
    """Unnormalised Walsh-Hadamard transform in place (``graph_sampler.py:90-93``)."""
    for q in range(int(math.log2(len(v)))):
        apply_one(v, HADAMARD, q)


def statevector(g, u):
    """(x)_q U_q |G> for all 2^n basis states (FP64; n <= ~26)."""
    v = graph_vector(g)
    for q in range(len(g)):
        apply_one(v, np.asarray(u[q]), q)
    return v


def conditional(g, u, A, B, outB):
    """Unnormalised A-vector given x_B = outB, and the B marginal (``graph_sampler.py:95-109``)."""
    g = np.asarray(g)
    mb = len(B)
    ids = np.arange(1 << mb, dtype=np.uint64)
    v = np.ones(1 << mb, dtype=np.complex128)
    for i, b in enumerate(B):
        v *= np.asarray(u[b])[outB[i], ((ids >> np.uint64(i)) & np.uint64(1)).astype(np.int64)]
    quadratic_phase(v, g[np.ix_(B, B)])
    walsh(v)
    ida = np.arange(1 << len(A), dtype=np.uint64)
    mapped = np.zeros_like(ida)
    for i, a in enumerate(A):
        mask = sum(1 << j for j, b in enumerate(B) if g[a, b])
        mapped ^= ((ida >> np.uint64(i)) & np.uint64(1)) * np.uint64(mask)
    va = v[mapped.astype(np.int64)] / (2.0 ** (len(g) / 2))
    quadratic_phase(va, g[np.ix_(A, A)])
    for i, a in enumerate(A):
        apply_one(va, np.asarray(u[a]), i)
    norm = float(np.vdot(va, va).real)
    return va, norm


# ----------------------------------------------------------------------------- Fourier-covariant sampler
def covariant_init(g, u, A, B, outB):
    """Initial vector of the covariant sampler before any transform
    (``fourier_covariant_sampler.py:66-70``): v[z] = 2^{-m/2} (-1)^{q_B(b)} prod_j U_Bj[out_j, b_j], b = N z."""
    g = np.asarray(g)
    m = len(A)
    N = gf2_inverse(g[np.ix_(B, A)]).T
    z = np.arange(1 << m, dtype=np.uint64)
    b = map_indices(z, N)
    v = np.full(1 << m, 2.0 ** (-m / 2), dtype=np.complex128)
    for j, site in enumerate(B):
        v *= np.asarray(u[site])[outB[j], ((b >> np.uint64(j)) & np.uint64(1)).astype(np.int64)]
    v *= phase_for_ids(b, g[np.ix_(B, B)])
    return v


def cpu_covariant(g, u, A, B, outB):
    """Normalised conditional A-state by Fourier covariance (``fourier_covariant_sampler.py:64-74``)."""
    g = np.asarray(g)
    v = covariant_init(g, u, A, B, outB)
    walsh(v)
    quadratic_phase(v, g[np.ix_(A, A)])
    for j, site in enumerate(A):
        apply_one(v, np.asarray(u[site]), j)
    return v


def cpu_deferred(g, u, A, B, outB):
    """State before and after the terminal unitary on the top A bit
    (``deferred_global_sampler.py:93-107``)."""
    g = np.asarray(g)
    m = len(A)
    N = gf2_inverse(g[np.ix_(B, A)]).T
    ids = np.arange(1 << (m - 1), dtype=np.uint64)
    halves = []
    for bit in (0, 1):
        z = ids | (np.uint64(bit) << np.uint64(m - 1))
        b = map_indices(z, N)
        v = np.full(len(ids), 2.0 ** (-m / 2), dtype=np.complex128)
        for j, site in enumerate(B):
            v *= np.asarray(u[site])[outB[j], ((b >> np.uint64(j)) & np.uint64(1)).astype(np.int64)]
        v *= phase_for_ids(b, g[np.ix_(B, B)])
        halves.append(v)
    raw = np.concatenate((halves[0] + halves[1], halves[0] - halves[1]))
    for bit in (0, 1):
        walsh(raw[bit * len(ids):(bit + 1) * len(ids)])
    quadratic_phase(raw, g[np.ix_(A, A)])
    for j, site in enumerate(A[:-1]):
        apply_one(raw, np.asarray(u[site]), j)
    final = raw.copy()
    apply_one(final, np.asarray(u[A[-1]]), m - 1)
    return raw, final


def cpu_shards(g, u, A, B, outB):
    """The two halves (top A bit = shard) of the state before the terminal unitary, each
    computed with shard-local operations only: the reference's two-device split
    (``np.split`` emulation of ``fourier_fused_sampler.py:161-169``) with the top bit's Walsh
    factor folded into the initialisation (``initcov_global``,
    ``deferred_global_sampler.py:23-37``); the q_A phase uses the global index."""
    g = np.asarray(g)
    m = len(A)
    N = gf2_inverse(g[np.ix_(B, A)]).T
    ids = np.arange(1 << (m - 1), dtype=np.uint64)
    inits = []
    for bit in (0, 1):
        b = map_indices(ids | (np.uint64(bit) << np.uint64(m - 1)), N)
        v = np.full(len(ids), 2.0 ** (-m / 2), dtype=np.complex128)
        for j, site in enumerate(B):
            v *= np.asarray(u[site])[outB[j], ((b >> np.uint64(j)) & np.uint64(1)).astype(np.int64)]
        v *= phase_for_ids(b, g[np.ix_(B, B)])
        inits.append(v)
    shards = [inits[0] + inits[1], inits[0] - inits[1]]
    for s, v in enumerate(shards):
        walsh(v)
        v *= phase_for_ids(ids | (np.uint64(s) << np.uint64(m - 1)), g[np.ix_(A, A)])
        for j, site in enumerate(A[:-1]):
            apply_one(v, np.asarray(u[site]), j)
    return shards


# ----------------------------------------------------------------------------- LUT specialisation
def transformed_quadratic(graph_B, N):
    """q(N z) = sum_{i<j} Q_ij z_i z_j + ell . z over GF(2) (``init_specialization.py:53-59``)."""
    upper = np.triu(np.asarray(graph_B, dtype=np.int64), 1)
    Nm = np.asarray(N, dtype=np.int64)
    P = (Nm.T @ upper @ Nm) & 1
    linear = np.diag(P).astype(np.uint8).copy()
    Q = np.triu(P ^ P.T, 1).astype(np.uint8)
    return Q, linear


def specialization_tables(g, A, B, chunk_bits=8):
    """Chunk lookup tables z-chunk -> (b XOR, phase mask | inner parity << 63)
    (``init_specialization.py:160-189``).  Returns (tables[chunks, 2^chunk_bits, 2], N, Q, linear_mask)."""
    g = np.asarray(g, dtype=np.uint8)
    m = len(B)
    N = gf2_inverse(g[np.ix_(B, A)]).T
    Q, linear = transformed_quadratic(g[np.ix_(B, B)], N)
    linear_mask = sum(int(bit) << i for i, bit in enumerate(linear))
    q_rows = [int(x) for x in row_masks(Q)]
    n_cols = [int(x) for x in row_masks(N.T)]
    chunks = math.ceil(m / chunk_bits)
    lut = np.zeros((chunks, 1 << chunk_bits, 2), dtype=np.uint64)
    for c in range(chunks):
        lo, hi = c * chunk_bits, min(m, (c + 1) * chunk_bits)
        above = ((1 << m) - 1) ^ ((1 << hi) - 1)
        for code in range(1 << (hi - lo)):
            z = code << lo
            b_xor = 0
            cross = 0
            inner = bin(z & linear_mask).count("1") & 1
            for j in range(lo, hi):
                if z >> j & 1:
                    b_xor ^= n_cols[j]
                    cross ^= q_rows[j] & above
                    inner ^= bin(z & q_rows[j]).count("1") & 1
            lut[c, code, 0] = b_xor
            lut[c, code, 1] = cross | (inner << 63)
    return lut, N, Q, linear_mask


def specialization_map_and_phase(lut, ids, chunk_bits=8):
    """b = N z and (-1)^{q_B(b)} from the chunk tables (``init_specialization.py:117-130``)."""
    ids = np.asarray(ids, dtype=np.uint64)
    b = np.zeros_like(ids)
    pm = np.zeros_like(ids)
    marked = ids | np.uint64(1 << 63)
    lowmask = np.uint64((1 << chunk_bits) - 1)
    for c in range(lut.shape[0]):
        code = ((ids >> np.uint64(c * chunk_bits)) & lowmask).astype(np.int64)
        b ^= lut[c, code, 0]
        pm ^= lut[c, code, 1] & marked
    return b, 1.0 - 2.0 * parity64(pm).astype(np.float64)


def specialization_weight_table(unitary, outB, m):
    """Table[k, h] = 2^{-m/2} U00^n00 U01^n01 U10^n10 U11^n11 indexed by popcounts
    (``init_specialization.py:98-115``)."""
    r = int(sum(int(x) for x in outB))
    powers = [np.power(complex(a), np.arange(m + 1)) for a in np.asarray(unitary).flat]
    table = np.zeros((m + 1, m + 1), dtype=np.complex128)
    for k in range(m + 1):
        for h in range(max(0, r + k - m), min(r, k) + 1):
            n00, n01, n10, n11 = m - r - k + h, k - h, r - h, h
            table[k, h] = 2.0 ** (-m / 2) * powers[0][n00] * powers[1][n01] * powers[2][n10] * powers[3][n11]
    return table


# ----------------------------------------------------------------------------- chain-rule sampling
def chain_conditionals(probs, order, bits):
    """p(x_{v_j} = 1 | x_{v_0..v_{j-1}}) for every position j of a bitstring, from the full
    probability vector (qubit q = index bit q).  Exact FP64 oracle for the scan chain rule."""
    n = len(order)
    idx = np.arange(len(probs), dtype=np.int64)
    alive = np.ones(len(probs), dtype=bool)
    out = np.zeros(n)
    for j, v in enumerate(order):
        tot = probs[alive].sum()
        one = probs[alive & (((idx >> v) & 1) == 1)].sum()
        out[j] = one / tot
        alive &= ((idx >> v) & 1) == int(bits[v])
    return out


def chain_sample(probs, order, uniforms):
    """Bitstring drawn position by position with x_v = 0 iff u * (M0 + M1) < M0, the
    rule of the GPU chain sampler, given one uniform per position."""
    n = len(order)
    idx = np.arange(len(probs), dtype=np.int64)
    alive = np.ones(len(probs), dtype=bool)
    bits = np.zeros(n, dtype=np.uint8)
    margins = np.zeros(n)
    for j, v in enumerate(order):
        m1 = probs[alive & (((idx >> v) & 1) == 1)].sum()
        m0 = probs[alive].sum() - m1
        x = 0 if uniforms[j] * (m0 + m1) < m0 else 1
        margins[j] = abs(uniforms[j] * (m0 + m1) - m0) / (m0 + m1)
        bits[v] = x
        alive &= ((idx >> v) & 1) == x
    return bits, margins
