"""Circuit front end (OpenQASM 2 -> graph + per-qubit unitaries) against a direct
statevector run of the same circuit (oracle/circuit.py).

* Random circuits of Clifford gates (h s sdg x y z sx sxdg id cx cz swap) followed by
  single-qubit tails (tdg, rz, u3, h): the derived (graph, unitaries) give the circuit's
  output distribution to 1e-12.
* |+>^n, CZ on every edge, then single-qubit gates: the graph is recovered exactly and
  the unitaries are the tails (the reference's RGS circuits have this form).
* QASM text with angle expressions parses to the same circuit; errors are ValueError.
"""
import math

import numpy as np
import pytest

from oracle import circuit
from oracle import graph_state as gs

CLIFF = ["h", "s", "sdg", "x", "y", "z", "sx", "sxdg", "id"]


def _random_circuit(rng, n):
    gates = []
    for _ in range(int(rng.integers(0, 6 * n + 1))):
        if n > 1 and rng.random() < 0.4:
            a, b = rng.choice(n, 2, replace=False)
            gates.append((str(rng.choice(["cx", "cz", "swap"])), (), [int(a), int(b)]))
        else:
            gates.append((str(rng.choice(CLIFF)), (), [int(rng.integers(n))]))
    for q in range(n):
        for _ in range(int(rng.integers(0, 3))):
            k = int(rng.integers(4))
            if k == 0:
                gates.append(("tdg", (), [q]))
            elif k == 1:
                gates.append(("rz", (float(rng.uniform(-3, 3)),), [q]))
            elif k == 2:
                gates.append(("u3", tuple(float(x) for x in rng.uniform(-3, 3, 3)), [q]))
            else:
                gates.append(("h", (), [q]))
    return gates


@pytest.mark.parametrize("seed", range(4))
def test_random_circuits_match_statevector(pkg, seed):
    fe = pkg.frontend
    rng = np.random.default_rng(seed)
    for _ in range(60):
        n = int(rng.integers(1, 9))
        gates = _random_circuit(rng, n)
        g, u = fe.circuit_to_graph(n, gates)
        assert np.array_equal(g, g.T) and not np.any(np.diag(g))
        ref = np.abs(circuit.run(n, gates, fe.gate_matrix)) ** 2
        got = np.abs(gs.statevector(g, u)) ** 2
        assert np.abs(ref - got).max() < 1e-12


def test_graph_state_circuit_recovers_graph(pkg):
    fe = pkg.frontend
    rng = np.random.default_rng(11)
    n = 10
    g0 = pkg.instances.regular3(n, rng)
    gates = [("h", (), [q]) for q in range(n)]
    gates += [("cz", (), [int(a), int(b)]) for a, b in pkg.edges_from_graph(g0)]
    angles = rng.uniform(-3, 3, (n, 3))
    gates += [("u3", tuple(float(x) for x in angles[q]), [q]) for q in range(n)]
    g, u = fe.circuit_to_graph(n, gates)
    assert np.array_equal(g, g0)
    for q in range(n):
        m = fe.gate_matrix("u3", angles[q])
        # Equal up to a global phase per qubit.
        k = np.vdot(m.ravel(), u[q].ravel())
        assert abs(abs(k) - 2) < 1e-12


def test_qasm_text(pkg):
    fe = pkg.frontend
    text = """OPENQASM 2.0;
include "qelib1.inc";
qreg q[4];
creg c[4];
h q[0]; h q[1];
sx q[2];
cx q[0],q[2];
cz q[1], q[3];
s q[3];
swap q[2],q[3];
rz(pi/2) q[1];
cz q[1],q[2];
tdg q[0];
rz(-3*pi/8) q[1];
u3(0.3, -pi/4, 2*pi/3) q[2];
ry(pi/5) q[3];
barrier q;
measure q -> c;
"""
    n, gates = fe.parse_qasm(text)
    assert n == 4 and len(gates) == 13
    assert gates[10] == ("rz", (-3 * math.pi / 8,), [1])
    g, u = fe.circuit_to_graph(n, gates)
    ref = np.abs(circuit.run(n, gates, fe.gate_matrix)) ** 2
    assert np.abs(ref - np.abs(gs.statevector(g, u)) ** 2).max() < 1e-12


def test_errors(pkg):
    fe = pkg.frontend
    with pytest.raises(ValueError):  # non-Clifford before an entangler on the same qubit
        fe.circuit_to_graph(2, [("t", (), [0]), ("cz", (), [0, 1])])
    with pytest.raises(ValueError):
        fe.circuit_to_graph(2, [("ccx", (), [0, 1])])
    with pytest.raises(ValueError):
        fe.parse_qasm("qreg q[2];\nh q[3];")
    with pytest.raises(ValueError):
        fe.parse_qasm("qreg q[2];\nrz(__import__('os')) q[0];")
    # rz by a multiple of pi/2 is Clifford and may precede an entangler.
    g, u = fe.circuit_to_graph(2, [("h", (), [0]), ("rz", (math.pi / 2,), [0]), ("cx", (), [0, 1])])
    ref = np.abs(circuit.run(2, [("h", (), [0]), ("rz", (math.pi / 2,), [0]), ("cx", (), [0, 1])],
                             fe.gate_matrix)) ** 2
    assert np.abs(ref - np.abs(gs.statevector(g, u)) ** 2).max() < 1e-12


@pytest.mark.gpu
def test_engine_on_front_end_output(pkg):
    """16-qubit circuits through the front end and the complex128 scan: p(x) of random
    strings equals the circuit's statevector."""
    fe = pkg.frontend
    rng = np.random.default_rng(7)
    for _ in range(3):
        n = 16
        gates = _random_circuit(rng, n)
        g, u = fe.circuit_to_graph(n, gates)
        order = rng.permutation(n).tolist()
        so = pkg.ScanOracle(g, u, order, fp64=True)
        bits = pkg.instances.uniform_bits(200, n, rng)
        ref = np.abs(circuit.run(n, gates, fe.gate_matrix)) ** 2
        idx = (bits.astype(np.int64) << np.arange(n)).sum(axis=1)
        p = so.probabilities(bits)
        assert np.allclose(p, ref[idx], rtol=1e-10, atol=1e-15)
