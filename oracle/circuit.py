"""Plain statevector simulation of a small gate-list circuit (test infrastructure only).

Checks the circuit front end: the (graph, unitaries) it derives must give the same output
distribution as running the circuit itself.  Qubit q is bit q of the basis index, as in
the reference (``W/graph_sampler.py:1``).  Gate matrices come from the front end's
``gate_matrix`` table; two-qubit gates are written out here.
"""
import numpy as np


def apply_1q(v, m, q, n):
    t = v.reshape((2,) * n)          # axis n-1-q is qubit q (C order, qubit 0 = last axis)
    ax = n - 1 - q
    t = np.moveaxis(t, ax, 0)
    t = np.tensordot(m, t, axes=([1], [0]))
    return np.moveaxis(t, 0, ax).reshape(-1)


def run(n, gates, gate_matrix):
    """|psi> = circuit |0^n>; gates as (name, args, qubits)."""
    v = np.zeros(1 << n, dtype=complex)
    v[0] = 1.0
    idx = np.arange(1 << n)
    for name, args, qs in gates:
        if len(qs) == 1:
            v = apply_1q(v, gate_matrix(name, args), qs[0], n)
        elif name == "cz":
            a, b = qs
            v = np.where(((idx >> a) & 1) & ((idx >> b) & 1), -v, v)
        elif name == "cx":
            a, b = qs
            flip = idx ^ (1 << b)
            v = np.where((idx >> a) & 1, v[flip], v)
        elif name == "swap":
            a, b = qs
            ba, bb = (idx >> a) & 1, (idx >> b) & 1
            src = idx ^ ((ba ^ bb) << a) ^ ((ba ^ bb) << b)
            v = v[src]
        else:
            raise ValueError(name)
    return v
