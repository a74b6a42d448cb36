"""The CPU oracle pinned against the reference's own known-answer tests,
restated (their file:line is in each test name's docstring), against the
golden fixtures and against the independent numpy simulator."""
from __future__ import annotations

import math

import numpy as np
import pytest

import numpy_sim

pytestmark = pytest.mark.filterwarnings("ignore")


def test_chacha_block_matches_rfc8439_vectors(oracle, golden):
    for v in golden["chacha20"]:
        assert oracle.chacha_block(v["key"], v["counter"], v["rounds"]) == v["words"]


def test_golden_circuits(oracle, golden):
    for fx in golden["circuits"]:
        n = fx["n"]
        s = oracle.StateVector(n)
        s.run(oracle.Circuit(fx["text"]), oracle.StdRng(0))
        want = np.zeros(1 << n, dtype=complex)
        want[fx["indices"]] = [complex(a, b) for a, b in fx["amplitudes"]]
        got = s.to_vector()
        assert np.abs(got - want).max() < 1e-12, fx["name"]


def test_ghz_exact_and_float(oracle):
    """src/state/vector.rs:580-633 (the C64 half)."""
    c = oracle.Circuit("QUBITS 3\nH 0\nCX 0 1\nCX 1 2\n")
    f = oracle.StateVector(3)
    rng = oracle.StdRng(1)
    f.run(c, rng)
    v = f.to_vector()
    r = 2 ** -0.5
    assert abs(v[0] - r) < 1e-14 and abs(v[7] - r) < 1e-14
    assert np.all(np.abs(v[1:7]) == 0)
    assert abs(f.expectation("X0*X1*X2") - 1) < 1e-14
    assert abs(f.expectation("Z0*Z1") - 1) < 1e-14
    assert abs(f.expectation("Z0")) < 1e-14
    zeros = 0
    for _ in range(200):
        s = f.clone()
        b = s.measure("Z0", rng)
        b1 = s.measure("Z1", rng)
        assert b == b1
        zeros += not b
    assert 60 <= zeros <= 140
    assert set(int(x) for x in f.sample(rng, 100)) <= {0, 7}
    p = f.clone()
    w = p.project_raw(0, 1, 0, True)
    assert abs(w.real - 0.5) < 1e-15
    p.normalize()
    assert abs(p.to_vector()[7] - 1) < 1e-15


def test_non_clifford_matches_matrix(oracle, golden):
    """src/state/vector.rs:635-654: run agrees with column 0 of the circuit unitary."""
    text = "QUBITS 2\nH 0\nH 1\nT 0\nCS 0 1\nSQRT_X 1\nRZ(0.7) 0\n"
    s = oracle.StateVector(2)
    s.run(oracle.Circuit(text), oracle.StdRng(0))
    u = np.eye(4, dtype=complex)
    for col in range(4):
        st = numpy_sim.NumpyState(2)
        st.v = u[:, col].copy()
        for line in text.splitlines()[1:]:
            toks = line.split()
            head = toks[0]
            name, args = (head.split("(")[0], head[head.index("(") + 1 : -1].split(",")) if "(" in head else (head, [])
            st.apply_line(name, args, [int(t) for t in toks[1:]])
        if col == 0:
            assert np.abs(s.to_vector() - st.v).max() < 1e-12


def _naive_apply(amp, m, qubits):
    """The obvious O(4^k 2^n) application (src/state/vector.rs:665-683)."""
    k = len(qubits)
    out = np.zeros_like(amp)
    idx = np.arange(amp.size)
    local = np.zeros(amp.size, dtype=np.int64)
    for j, q in enumerate(qubits):
        local |= ((idx >> q) & 1) << j
    for b in range(1 << k):
        w = idx.copy()
        for j, q in enumerate(qubits):
            w = (w & ~(1 << q)) | (((b >> j) & 1) << q)
        out += m[local, b] * amp[w]
    return out


def test_fiber_kernel_matches_naive_on_high_and_low_qubits(oracle):
    """src/state/vector.rs:685-757, including Pauli expectation/apply/project."""
    rng = np.random.default_rng(8)
    n = 15
    v = oracle.StateVector(n)
    v.set_amplitudes(rng.random(1 << n) - 0.5 + 1j * (rng.random(1 << n) - 0.5))
    for trial in range(12):
        k = 1 + trial % 3
        qs = []
        while len(qs) < k:
            q = int(rng.integers(12, n)) if rng.random() < 0.5 else int(rng.integers(0, 12))
            if q not in qs:
                qs.append(q)
        m = rng.random((1 << k, 1 << k)) + 1j * rng.random((1 << k, 1 << k))
        want = _naive_apply(v.to_vector(), m, qs)
        v.apply_matrix(m, qs)
        assert np.abs(v.to_vector() - want).max() < 1e-9, (trial, qs)
        v.scale(1 / math.sqrt(v.norm_sq().real))
    for trial in range(10):
        x = int(rng.integers(0, 1 << n))
        z = int(rng.integers(0, 1 << n))
        ph = bin(x & z).count("1") % 4  # letter phase 0: the Hermitian product of letters
        if trial % 3 == 0:
            ph = (ph + 2) % 4
        a = v.to_vector()
        pv = numpy_sim.pauli_matrix_action(a, n, x, z, ph)
        assert abs(v.expectation_raw(x, z, ph) - np.vdot(a, pv)) < 1e-9
        u = v.clone()
        u.apply_pauli_raw(x, z, ph)
        assert np.abs(u.to_vector() - pv).max() < 1e-12
        w = v.clone()
        b = bool(rng.integers(0, 2))
        w.project_raw(x, z, ph, b)
        sgn = -1.0 if b else 1.0
        assert np.abs(w.to_vector() - (a + sgn * pv) * 0.5).max() < 1e-12


def test_one_pass_sampling_follows_the_born_rule_across_blocks(oracle):
    """src/state/vector.rs:767-800."""
    n = 14
    i = np.arange(1 << n)
    amps = np.where(i % 4099 == 7, 3.0, 0.01 * (i % 13)).astype(complex)
    v = oracle.StateVector.from_amplitudes(amps)
    shots = 200_000
    s = v.sample(oracle.StdRng(2), shots).astype(np.int64)
    total = np.sum(np.abs(amps) ** 2)
    counts = np.bincount(s, minlength=1 << n)
    for k in range(7, 1 << n, 4099):
        p = abs(amps[k]) ** 2 / total
        f = counts[k] / shots
        assert abs(f - p) < 6 * math.sqrt(p * (1 - p) / shots), k
    assert np.all((s % 13 != 0) | (s % 4099 == 7))


def test_clifford_t_backends_and_expectations(oracle, golden):
    """tests/backends.rs:35-75 (the StateVector side): amplitudes and four Pauli expectations."""
    fx = next(c for c in golden["circuits"] if c["name"].startswith("clifford_t"))
    v = oracle.StateVector(4)
    v.run(oracle.Circuit(fx["text"]), oracle.StdRng(0))
    a = v.to_vector()
    ref = numpy_sim.run_text(fx["text"])
    assert np.abs(a - ref).max() < 1e-9
    for text, (x, z, ph) in {
        "X0*Z1": (1, 2, 0),
        "Y2": (4, 4, 1),
        "Z0*Z1*Z2*Z3": (0, 15, 0),
        "X3": (8, 0, 0),
    }.items():
        want = np.vdot(ref, numpy_sim.pauli_matrix_action(ref, 4, x, z, ph))
        assert abs(v.expectation(text) - want) < 1e-9, text


def test_clifford_circuit_with_measurements(oracle):
    """tests/backends.rs:77-107 (StateVector): first outcome deterministic, record consistent."""
    text = "QUBITS 3\nH 0\nCX 0 1\nCX 1 2\nS 2\nMPP Z0*Z1\nMPP X0*X1*X2\nM 0\n"
    v = oracle.StateVector(3)
    rec = v.run(oracle.Circuit(text), oracle.StdRng(3))
    assert rec[0] is False
    z0 = v.expectation("Z0").real / v.norm_sq().real
    assert abs(z0 - (-1.0 if rec[2] else 1.0)) < 1e-12


def test_sampling_statistics(oracle):
    """tests/backends.rs:138-179 (StateVector histogram within 4 sqrt(E) + 5)."""
    text = "QUBITS 3\nH 0\nCX 0 1\nT 1\nH 1\nCX 1 2\n"
    v = oracle.StateVector(3)
    rng = oracle.StdRng(42)
    v.run(oracle.Circuit(text), rng)
    shots = 600
    h = np.bincount(v.sample(rng, shots).astype(np.int64), minlength=8)
    probs = np.abs(v.to_vector()) ** 2 / v.norm_sq().real
    for x in range(8):
        e = probs[x] * shots
        assert abs(h[x] - e) < 4 * math.sqrt(max(e, 1.0)) + 5


def test_kron_index_convention(oracle):
    """tests/backends.rs:181-201: amplitude x_a + 8 x_b."""
    va, vb = oracle.StateVector(3), oracle.StateVector(2)
    rng = oracle.StdRng(11)
    va.run(oracle.Circuit("QUBITS 3\nH 0 1\nT 0\nCX 0 2\nS 2\nH 2\nCCZ 0 1 2\n"), rng)
    vb.run(oracle.Circuit("QUBITS 2\nH 0\nCX 0 1\nT_DAG 1\nH 1\n"), rng)
    k = va.kron(vb).to_vector()
    a, b = va.to_vector(), vb.to_vector()
    for xa in range(8):
        for xb in range(4):
            assert abs(k[xa + 8 * xb] - a[xa] * b[xb]) < 1e-12


NAMED = ["I", "X", "Y", "Z", "H", "S", "S_DAG", "SQRT_X", "SQRT_X_DAG", "SQRT_Y", "SQRT_Y_DAG", "T", "T_DAG",
         "CX", "CY", "CZ", "SWAP", "CS", "CS_DAG", "CCZ", "CCX", "PHASE(3,4)", "CPHASE(1,3)"]


@pytest.mark.parametrize("name", NAMED)
def test_gate_views_agree_with_matrices(oracle, name):
    """src/gate.rs:904-984: unitary, dagger, and agreement with independent definitions."""
    k = {"CX": 2, "CY": 2, "CZ": 2, "SWAP": 2, "CS": 2, "CS_DAG": 2, "CPHASE(1,3)": 2, "CCZ": 3, "CCX": 3}.get(name, 1)
    text = f"QUBITS {k}\n{name} " + " ".join(str(q) for q in range(k)) + "\n"
    m = oracle.gate_matrix(text)
    d = 1 << k
    assert np.abs(m @ m.conj().T - np.eye(d)).max() < 1e-12
    md = oracle.gate_matrix(text, dagger=True)
    assert np.abs(md - m.conj().T).max() < 1e-12
    head = name.split("(")[0]
    args = name[name.index("(") + 1 : -1].split(",") if "(" in name else []
    assert np.abs(m - numpy_sim.named_matrix(head, args)).max() < 1e-12


def test_root_of_unity_and_sqrt2_pow_constants(oracle):
    """src/scalar.rs:443-468 through the phase gates: PHASE(k,b) = diag(1, exp(2 pi i k/2^b))."""
    for bits in range(1, 6):
        for kk in range(1 << bits):
            m = oracle.gate_matrix(f"QUBITS 1\nPHASE({kk},{bits}) 0\n")
            assert abs(m[1, 1] - np.exp(2j * np.pi * kk / (1 << bits))) < 1e-14
    m = oracle.gate_matrix("QUBITS 1\nH 0\n")
    assert m[0, 0].real == 0.5 * math.sqrt(2.0)


@pytest.mark.parametrize("n,depth,seed", [(6, 5, 3), (10, 8, 1), (12, 6, 7)])
def test_oracle_matches_numpy_on_random_layers(oracle, n, depth, seed):
    text = oracle.random_circuit_text(n, depth, seed)
    s = oracle.StateVector(n)
    s.run(oracle.Circuit(text), oracle.StdRng(0))
    assert np.abs(s.to_vector() - numpy_sim.run_text(text)).max() < 1e-12


def test_oracle_matches_numpy_on_reversible_family(oracle):
    text = oracle.reversible_circuit_text(11, 60, 4)
    s = oracle.StateVector(11)
    s.run(oracle.Circuit(text), oracle.StdRng(0))
    a = s.to_vector()
    assert np.abs(a - numpy_sim.run_text(text)).max() < 1e-12
    idx, amp = oracle.sparse_run(text)
    assert np.array_equal(np.flatnonzero(a), idx.astype(np.int64))
    assert np.array_equal(a[idx.astype(np.int64)], amp)  # bit-identical arithmetic


def test_parse_errors(oracle):
    """src/circuit.rs:772-785."""
    for bad in ["CX 0", "QUBITS 1\nH 3", "FOO 1"]:
        with pytest.raises(oracle.OracleError):
            oracle.Circuit(bad)
    c = oracle.Circuit("H 0\nCX 0 1 1 2\nT 2\nPHASE(3,4) 1\nM 0\nMX 1\nMPP X0*Z2\nR 2\nTICK\n")
    assert (c.num_qubits, c.num_gates, c.num_measurements) == (3, 5, 3)


def test_trajectory_is_deterministic(oracle):
    a = oracle.trajectory(5)
    b = oracle.trajectory(5)
    assert a == b and 16 <= a[0] <= 22 and len(a[2]) == a[0]
