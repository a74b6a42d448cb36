"""Tiled passes of the plain path: runs of gates applied to shared-memory tiles
give the same amplitudes as the gate-by-gate kernels (bit for bit: each gate
keeps its kernel's arithmetic) and agree with the oracle within 1e-12, for
every gate form a pass carries (1- to 3-qubit dense matrices, diagonal
constants and tables, pair swaps, phase polynomials) and the forms it leaves
to their own kernels (other permutation tables)."""
from __future__ import annotations

import random

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12

ONE = ["H", "S", "S_DAG", "T", "T_DAG", "SQRT_X", "SQRT_X_DAG", "SQRT_Y", "X", "Y", "Z", "RX(0.37)", "RY(1.3)",
       "RZ(2.1)", "PHASE(3,4)"]
TWO = ["CX", "CY", "CZ", "SWAP", "CS", "CS_DAG", "CPHASE(1,3)"]
THREE = ["CCX", "CCZ"]


def _mixed_text(n, gates, seed):
    r = random.Random(seed)
    lines = [f"QUBITS {n}"]
    for _ in range(gates):
        u = r.random()
        if u < 0.5:
            lines.append(f"{r.choice(ONE)} {r.randrange(n)}")
        elif u < 0.85:
            a, b = r.sample(range(n), 2)
            lines.append(f"{r.choice(TWO)} {a} {b}")
        elif u < 0.95:
            a, b, c = r.sample(range(n), 3)
            lines.append(f"{r.choice(THREE)} {a} {b} {c}")
        else:
            qs = r.sample(range(n), 3)
            lines.append(f"DIAG(3;1;1:1;3:2,4;5:1,2,4) {' '.join(map(str, qs))}")
    return "\n".join(lines) + "\n"


def _run_both(nb, text, n, precision, seed=0):
    c = nb.Circuit.parse(text)
    a = nb.GpuStateVector(n, precision)
    a.set_tile_passes(False)
    b = nb.GpuStateVector(n, precision)
    for s in (a, b):  # the second run of a circuit is captured as a graph: run it twice
        s.run(c, nb.StdRng(seed))
        s.set_basis(0)
        s.run(c, nb.StdRng(seed))
    return a, b


@pytest.mark.parametrize("n", [10, 14, 17, 21])
def test_random_layers_equal_gate_by_gate(nb, oracle, n):
    text = oracle.random_circuit_text(n, 8, n, 0.0, 0, 0)
    a, b = _run_both(nb, text, n, nb.C128)
    va, vb = a.to_vector(), b.to_vector()
    assert np.array_equal(va, vb)
    o = oracle.StateVector(n)
    o.run(oracle.Circuit(text), oracle.StdRng(0))
    assert np.abs(vb - o.to_vector()).max() < TOL


@pytest.mark.parametrize("n,precision", [(13, 0), (18, 0), (16, 1)])
def test_mixed_gates_equal_gate_by_gate(nb, oracle, n, precision):
    text = _mixed_text(n, 300, 100 + n)
    a, b = _run_both(nb, text, n, precision)
    assert np.array_equal(a.to_vector(), b.to_vector())
    if precision == 0:
        o = oracle.StateVector(n)
        o.run(oracle.Circuit(text), oracle.StdRng(0))
        assert np.abs(b.to_vector() - o.to_vector()).max() < TOL


def test_reversible_family_equal_gate_by_gate(nb, oracle):
    n = 20
    text = oracle.reversible_circuit_text(n, 200, 9)
    a, b = _run_both(nb, text, n, nb.C128)
    assert np.array_equal(a.to_vector(), b.to_vector())


def test_dense_unitaries_in_runs(nb, oracle):
    """Circuits of Clifford and phase gates with 3-qubit DIAG and MONOMIAL tables
    between them: pair-swap monomials and diagonal tables join passes, other
    permutation tables run as their own kernels."""
    n = 15
    r = random.Random(4)
    lines = [f"QUBITS {n}"]
    for _ in range(120):
        u = r.random()
        if u < 0.5:
            lines.append(f"{r.choice(ONE)} {r.randrange(n)}")
        elif u < 0.7:
            qs = r.sample(range(n), 3)
            lines.append(f"MONOMIAL(1,3,4;2;2;0;1:1;3:2,4;0,0,0) {' '.join(map(str, qs))}")
        elif u < 0.85:
            qs = r.sample(range(n), 3)
            lines.append(f"MONOMIAL(2,1,4;0;1;0;0,0,0) {' '.join(map(str, qs))}")
        else:
            a, b = r.sample(range(n), 2)
            lines.append(f"{r.choice(TWO)} {a} {b}")
    text = "\n".join(lines) + "\n"
    a, b = _run_both(nb, text, n, nb.C128, seed=1)
    assert np.array_equal(a.to_vector(), b.to_vector())
    o = oracle.StateVector(n)
    o.run(oracle.Circuit(text), oracle.StdRng(1))
    assert np.abs(b.to_vector() - o.to_vector()).max() < TOL


def test_runs_between_measurements_and_noise(nb, oracle):
    n = 16
    text = oracle.random_circuit_text(n, 6, 3, 0.01, n - 4, n)
    text += "".join(f"H {q}\n" for q in range(n)) + "".join(f"T {q}\n" for q in range(n)) + "M 0 1\n"
    a, b = _run_both(nb, text, n, nb.C128, seed=5)
    assert np.array_equal(a.to_vector(), b.to_vector())
    rec_a = a.run(nb.Circuit.parse(text), nb.StdRng(6))
    rec_b = b.run(nb.Circuit.parse(text), nb.StdRng(6))
    assert rec_a == rec_b


def test_passes_are_used(nb, oracle):
    n = 20
    c = nb.Circuit.parse(oracle.random_circuit_text(n, 4, 1, 0.0, 0, 0))
    s = nb.GpuStateVector(n)
    s.profile(True)
    s.run(c, nb.StdRng(0))
    prof = s.profile_read()
    s.profile(False)
    assert prof.get("plain_pass", {}).get("launches", 0) >= 2, prof
    launches = sum(v["launches"] for v in prof.values())
    assert launches < c.num_gates // 4, (launches, c.num_gates)
