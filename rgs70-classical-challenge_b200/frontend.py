"""Circuit front end: an OpenQASM 2 circuit of Clifford gates followed by single-qubit
gates -> (graph, per-qubit unitaries) for the scan engine.

A circuit C on |0^n> whose two-qubit gates are Clifford is a stabilizer state S times
single-qubit gates V_q applied after each qubit's last two-qubit gate.  Every stabilizer
state is local-Clifford equivalent to a graph state: S = (x)_q L_q^dag |G>, so
p(x) = |<x| (x)_q V_q L_q^dag |G>|^2 -- exactly the engine's contraction with
u_q = V_q L_q^dag.  This replaces the reference's ``parse_qasm`` / ``Tableau.to_graph``
(whyihaveyou/rgs70-classical-challenge, ``W/graph_sampler.py:11-57, 111-132``) with any
number of qubits up to 128, the tail split per qubit (a qubit's single-qubit gates after
its last entangler), and a check that needs no Stim: the graph form is verified against
the tableau it came from.

The stabilizer tableau holds n generators as bit rows (x | z) and sign bits; gates act by
conjugation (Aaronson & Gottesman, Phys. Rev. A 70, 052328 (2004)).
"""
import ast
import math
import operator
import re

import numpy as np

__all__ = ["Tableau", "parse_qasm", "circuit_to_graph", "gate_matrix"]

_H = np.array([[1, 1], [1, -1]], dtype=complex) / math.sqrt(2)
_S = np.diag([1, 1j])
_CLIFFORD_1Q = {"id", "h", "s", "sdg", "x", "y", "z", "sx", "sxdg"}
_TWO_Q = {"cx", "cz", "swap"}


def _angle(expr):
    """Evaluate a QASM angle expression (numbers, pi, + - * / and parentheses)."""
    ops = {ast.Add: operator.add, ast.Sub: operator.sub, ast.Mult: operator.mul, ast.Div: operator.truediv,
           ast.USub: operator.neg, ast.UAdd: operator.pos, ast.Pow: operator.pow}

    def ev(node):
        if isinstance(node, ast.Expression):
            return ev(node.body)
        if isinstance(node, ast.Constant) and isinstance(node.value, (int, float)):
            return float(node.value)
        if isinstance(node, ast.Name) and node.id == "pi":
            return math.pi
        if isinstance(node, ast.BinOp) and type(node.op) in ops:
            return ops[type(node.op)](ev(node.left), ev(node.right))
        if isinstance(node, ast.UnaryOp) and type(node.op) in ops:
            return ops[type(node.op)](ev(node.operand))
        raise ValueError(f"unsupported angle expression: {expr!r}")
    return ev(ast.parse(expr.strip(), mode="eval"))


def gate_matrix(name, args=()):
    """2x2 matrix of a single-qubit gate (global phases as in the OpenQASM definitions)."""
    a = list(args)
    if name == "id":
        return np.eye(2, dtype=complex)
    if name == "h":
        return _H.copy()
    if name == "s":
        return _S.copy()
    if name == "sdg":
        return _S.conj().T
    if name == "t":
        return np.diag([1, np.exp(1j * math.pi / 4)])
    if name == "tdg":
        return np.diag([1, np.exp(-1j * math.pi / 4)])
    if name == "x":
        return np.array([[0, 1], [1, 0]], dtype=complex)
    if name == "y":
        return np.array([[0, -1j], [1j, 0]], dtype=complex)
    if name == "z":
        return np.diag([1, -1]).astype(complex)
    if name == "sx":
        return np.array([[1 + 1j, 1 - 1j], [1 - 1j, 1 + 1j]]) / 2
    if name == "sxdg":
        return np.array([[1 - 1j, 1 + 1j], [1 + 1j, 1 - 1j]]) / 2
    if name == "rz":
        return np.diag([np.exp(-0.5j * a[0]), np.exp(0.5j * a[0])])
    if name == "rx":
        c, s = math.cos(a[0] / 2), math.sin(a[0] / 2)
        return np.array([[c, -1j * s], [-1j * s, c]])
    if name == "ry":
        c, s = math.cos(a[0] / 2), math.sin(a[0] / 2)
        return np.array([[c, -s], [s, c]], dtype=complex)
    if name in ("p", "u1"):
        return np.diag([1, np.exp(1j * a[0])])
    if name in ("u", "u3"):
        th, ph, la = a
        return np.array([[math.cos(th / 2), -np.exp(1j * la) * math.sin(th / 2)],
                         [np.exp(1j * ph) * math.sin(th / 2), np.exp(1j * (ph + la)) * math.cos(th / 2)]])
    if name == "u2":
        return gate_matrix("u3", (math.pi / 2, a[0], a[1]))
    raise ValueError(f"unsupported gate {name!r}")


class Tableau:
    """Stabilizer generators of an n-qubit state: rows (x | z) and sign bits r."""

    def __init__(self, n):
        self.n = int(n)
        self.x = np.zeros((n, n), dtype=np.uint8)
        self.z = np.eye(n, dtype=np.uint8)
        self.r = np.zeros(n, dtype=np.uint8)

    # ------------------------------------------------------------------ gates (conjugation)
    def h(self, a):
        self.r ^= self.x[:, a] & self.z[:, a]
        self.x[:, a], self.z[:, a] = self.z[:, a].copy(), self.x[:, a].copy()

    def s(self, a):
        self.r ^= self.x[:, a] & self.z[:, a]
        self.z[:, a] ^= self.x[:, a]

    def apply(self, name, qs):
        a = qs[0]
        if name == "id":
            return
        if name == "h":
            self.h(a)
        elif name == "s":
            self.s(a)
        elif name == "sdg":
            for _ in range(3):
                self.s(a)
        elif name == "z":
            self.r ^= self.x[:, a]
        elif name == "x":
            self.r ^= self.z[:, a]
        elif name == "y":
            self.r ^= self.x[:, a] ^ self.z[:, a]
        elif name == "sx":  # H S H
            self.h(a)
            self.s(a)
            self.h(a)
        elif name == "sxdg":
            self.h(a)
            for _ in range(3):
                self.s(a)
            self.h(a)
        elif name == "cx":
            b = qs[1]
            self.r ^= self.x[:, a] & self.z[:, b] & (self.x[:, b] ^ self.z[:, a] ^ 1)
            self.x[:, b] ^= self.x[:, a]
            self.z[:, a] ^= self.z[:, b]
        elif name == "cz":
            b = qs[1]
            self.h(b)
            self.apply("cx", [a, b])
            self.h(b)
        elif name == "swap":
            b = qs[1]
            for c, t in ((a, b), (b, a), (a, b)):
                self.apply("cx", [c, t])
        else:
            raise ValueError(f"not a Clifford gate: {name!r}")

    # ------------------------------------------------------------------ row algebra
    def _mul_rows(self, i, j):
        """Row i <- row i * row j (Pauli product with its sign)."""
        x1, z1 = self.x[i].astype(np.int64), self.z[i].astype(np.int64)
        x2, z2 = self.x[j].astype(np.int64), self.z[j].astype(np.int64)
        # Phase exponent (in units of i) of each single-qubit product, summed.
        g = np.where((x1 == 1) & (z1 == 1), z2 - x2,
                     np.where((x1 == 1) & (z1 == 0), z2 * (2 * x2 - 1),
                              np.where((x1 == 0) & (z1 == 1), x2 * (1 - 2 * z2), 0)))
        tot = (2 * int(self.r[i]) + 2 * int(self.r[j]) + int(g.sum())) % 4
        if tot % 2:
            raise ArithmeticError("generators do not commute")
        self.r[i] = tot // 2
        self.x[i] ^= self.x[j]
        self.z[i] ^= self.z[j]

    def to_graph(self):
        """Local Cliffords L_q (2x2) and the adjacency G with (x)_q L_q |this> = |G> up to a
        global phase.  Works on a copy; the graph form is checked before returning."""
        t = Tableau(self.n)
        t.x, t.z, t.r = self.x.copy(), self.z.copy(), self.r.copy()
        n = self.n
        local = np.repeat(np.eye(2, dtype=complex)[None], n, axis=0)
        # Make the X block invertible (H where a column has no pivot) and reduce it to I.
        for col in range(n):
            piv = [i for i in range(col, n) if t.x[i, col]]
            if not piv:
                t.h(col)
                local[col] = _H @ local[col]
                piv = [i for i in range(col, n) if t.x[i, col]]
            if not piv:
                raise ArithmeticError("no pivot: the generators are dependent")
            p = piv[0]
            if p != col:
                for arr in (t.x, t.z):
                    arr[[col, p]] = arr[[p, col]]
                t.r[[col, p]] = t.r[[p, col]]
            for i in range(n):
                if i != col and t.x[i, col]:
                    t._mul_rows(i, col)
        if not np.array_equal(t.x, np.eye(n, dtype=np.uint8)):
            raise ArithmeticError("X block did not reduce to the identity")
        # Generator q is now X_q Z^{z_q}: clear Y on the diagonal (S^dag), then the signs (Z).
        for q in range(n):
            if t.z[q, q]:
                for _ in range(3):
                    t.s(q)
                local[q] = _S.conj().T @ local[q]
        for q in range(n):
            if t.r[q]:
                t.r ^= t.x[:, q]
                local[q] = np.diag([1, -1]) @ local[q]
        g = t.z.copy()
        if np.any(t.r) or not np.array_equal(g, g.T) or np.any(np.diag(g)):
            raise ArithmeticError("not in graph form")
        return g, local


def parse_qasm(text):
    """(n, gates) of an OpenQASM 2 text: gates as (name, float args, qubits)."""
    m = re.search(r"qreg\s+(\w+)\s*\[\s*(\d+)\s*\]\s*;", text)
    if not m:
        raise ValueError("no qreg declaration")
    reg, n = m.group(1), int(m.group(2))
    gates = []
    for raw in text.split(";"):
        line = raw.strip()
        if not line or line.startswith(("OPENQASM", "include", "qreg", "creg", "barrier", "measure", "//")):
            continue
        g = re.match(r"^(\w+)\s*(?:\(([^)]*)\))?\s+(.*)$", line, re.S)
        if not g:
            raise ValueError(f"cannot parse: {line!r}")
        name, args, ops = g.group(1).lower(), g.group(2), g.group(3)
        qs = [int(x) for x in re.findall(rf"{reg}\s*\[\s*(\d+)\s*\]", ops)]
        if not qs or any(q >= n for q in qs):
            raise ValueError(f"bad operands: {line!r}")
        vals = tuple(_angle(a) for a in args.split(",")) if args else ()
        gates.append((name, vals, qs))
    return n, gates


def _clifford_rz(theta):
    """rz(k pi / 2) as Clifford gates (up to a global phase), or None."""
    k = theta / (math.pi / 2)
    kr = round(k)
    if abs(k - kr) > 1e-12:
        return None
    return {0: [], 1: ["s"], 2: ["z"], 3: ["sdg"]}[kr % 4]


def circuit_to_graph(n, gates):
    """(g uint8 [n, n], u complex128 [n, 2, 2]) with p(x) = |<x| (x)_q u_q |G>|^2 for the
    circuit's output on |0^n>.  Single-qubit gates after a qubit's last two-qubit gate
    form its tail V_q; everything before must be Clifford."""
    last = [-1] * n
    for i, (name, _, qs) in enumerate(gates):
        if len(qs) == 2:
            if name not in _TWO_Q:
                raise ValueError(f"unsupported two-qubit gate {name!r}")
            for q in qs:
                last[q] = i
        elif len(qs) != 1:
            raise ValueError(f"unsupported gate arity: {name!r}")
    tab = Tableau(n)
    tail = np.repeat(np.eye(2, dtype=complex)[None], n, axis=0)
    for i, (name, args, qs) in enumerate(gates):
        if len(qs) == 2:
            tab.apply(name, qs)
            continue
        q = qs[0]
        if i > last[q]:
            tail[q] = gate_matrix(name, args) @ tail[q]
        elif name in _CLIFFORD_1Q:
            tab.apply(name, qs)
        elif name == "rz" and _clifford_rz(args[0]) is not None:
            for c in _clifford_rz(args[0]):
                tab.apply(c, qs)
        else:
            raise ValueError(f"non-Clifford gate {name!r} on qubit {q} before its last two-qubit gate")
    g, local = tab.to_graph()
    u = tail @ local.conj().transpose(0, 2, 1)
    return g, u
