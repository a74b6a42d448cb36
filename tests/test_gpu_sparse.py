"""The sparse form (``SparseVector<C64>``, src/state/sparse.rs) on the device,
against the CPU oracle: the dense FP64 restatement for registers small enough
to hold densely, and the sparse restatement for the reversible family.

Bars, as for the dense drop-in: amplitudes within 1e-12, nonzero index sets
bit-exact, measurement records identical for the same seeded StdRng, sampled
indices equal shot for shot to the reference's rule (cumulative weights in
entry order, one draw per shot).
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12

ONE_Q = ["H", "X", "Y", "Z", "S", "S_DAG", "T", "T_DAG", "SQRT_X", "SQRT_Y", "RX(0.7)", "RY(1.3)", "RZ(0.4)",
         "PHASE(1,3)"]
TWO_Q = ["CX", "CY", "CZ", "SWAP", "CS", "CPHASE(3,8)"]
THREE_Q = ["CCX", "CCZ"]


def random_gates(n, count, rng):
    """A random gate list in the spirit of the reference's sparse test (sparse.rs:457-488)."""
    lines = [f"QUBITS {n}"]
    for _ in range(count):
        r = rng.random()
        if r < 0.55 or n < 2:
            lines.append(f"{ONE_Q[rng.integers(len(ONE_Q))]} {rng.integers(n)}")
        elif r < 0.85 or n < 3:
            a, b = rng.choice(n, 2, replace=False)
            lines.append(f"{TWO_Q[rng.integers(len(TWO_Q))]} {a} {b}")
        else:
            a, b, c = rng.choice(n, 3, replace=False)
            lines.append(f"{THREE_Q[rng.integers(len(THREE_Q))]} {a} {b} {c}")
    return "\n".join(lines) + "\n"


def pauli_text(n, rng):
    return "".join("_XYZ"[rng.integers(4)] for _ in range(n))


def sorted_entries(s):
    k, a = s.entries()
    o = np.argsort(k)
    return k[o], a[o]


def test_random_gates_match_the_dense_vector(nb, oracle):
    """sparse.rs:490-539: amplitudes, <P>, projection weights, <a|b>, Paulis."""
    rng = np.random.default_rng(13)
    for trial in range(24):
        n = 3 + trial % 6
        text = random_gates(n, 30, rng)
        s = nb.GpuSparseVector(n)
        s.run(nb.Circuit.parse(text), nb.StdRng(0))
        v = oracle.StateVector(n)
        v.run(oracle.Circuit(text), oracle.StdRng(0))
        assert np.abs(s.to_vector() - v.to_vector()).max() < TOL, trial
        # the entries are the nonzero amplitudes, sorted after a normalisation
        k, a = sorted_entries(s)
        dense = v.to_vector()
        assert np.array_equal(k, np.flatnonzero(dense).astype(np.uint64))
        pt = pauli_text(n, rng)
        p = nb.Pauli.from_string(n, pt)
        assert abs(s.expectation(p) - v.expectation_raw(p.x, p.z, p.phase)) < 1e-10
        s2, v2 = s.clone(), v.clone()
        b = bool(rng.integers(2))
        if p.is_hermitian():
            assert abs(s2.project(p, b) - v2.project_raw(p.x, p.z, p.phase, b)) < 1e-10
            assert abs(s.inner(s2) - v.inner(v2)) < 1e-10
            assert np.abs(s2.to_vector() - v2.to_vector()).max() < TOL
        s3, v3 = s.clone(), v.clone()
        s3.apply_pauli(p)
        v3.apply_pauli_raw(p.x, p.z, p.phase)
        assert np.abs(s3.to_vector() - v3.to_vector()).max() < TOL
        assert abs(s.norm_sq() - v.norm_sq()) < 1e-12


def test_reversible_family_matches_the_sparse_restatement(nb, oracle):
    text = oracle.reversible_circuit_text(20, 400, 2)
    s = nb.GpuSparseVector(20)
    s.run(nb.Circuit.parse(text), nb.StdRng(0))
    idx, amp = oracle.sparse_run(text)
    k, a = sorted_entries(s)
    assert np.array_equal(k, idx)
    assert np.abs(a - amp).max() < TOL


def test_reversible_family_at_31_qubits(nb, oracle):
    """The C3 shape: n = 31, 2000 permutation and diagonal gates, 2^16 entries."""
    c = nb.Circuit.reversible(31, 2000, 1)
    s = nb.GpuSparseVector(31)
    s.run(c, nb.StdRng(0))
    idx, amp = oracle.sparse_run(c.to_text())
    assert s.num_entries() == idx.size == 1 << 16
    k, a = sorted_entries(s)
    assert np.array_equal(k, idx)
    assert np.abs(a - amp).max() < TOL
    assert abs(s.norm_sq().real - 1.0) < 1e-12


def test_measurements_noise_and_resets_match_the_dense_run(nb, oracle):
    rng = np.random.default_rng(5)
    for trial in range(6):
        n = 6 + trial
        body = random_gates(n, 40, rng).splitlines()[1:]
        body += ["DEPOLARIZE1(0.3) 1", "X_ERROR(0.5) 2", "DEPOLARIZE2(0.4) 0 3", "R 4"]
        body += random_gates(n, 10, rng).splitlines()[1:]
        body += [f"M {q}" for q in range(n)]
        text = f"QUBITS {n}\n" + "\n".join(body) + "\n"
        s = nb.GpuSparseVector(n)
        rec = s.run(nb.Circuit.parse(text), nb.StdRng(100 + trial))
        v = oracle.StateVector(n)
        rec_o = v.run(oracle.Circuit(text), oracle.StdRng(100 + trial))
        assert rec == rec_o, trial
        assert np.abs(s.to_vector() - v.to_vector()).max() < TOL


def test_sampling_follows_the_entry_order(nb, oracle):
    """sample (sparse.rs:407-424): the cumulative weights of the entries in their
    current (here unsorted) order, u = gen::<f64>() * total per shot."""
    rng = np.random.default_rng(3)
    text = random_gates(9, 25, rng) + "CX 0 5\nCCX 1 2 8\nSWAP 3 7\n"
    s = nb.GpuSparseVector(9)
    s.run(nb.Circuit.parse(text), nb.StdRng(0))
    got = s.sample(nb.StdRng(77), 500)
    k, a = s.entries()
    cum = np.cumsum(np.abs(a) ** 2)
    r = oracle.StdRng(77)
    want = []
    for _ in range(500):
        u = r.gen_f64() * cum[-1]
        want.append(int(k[min(int(np.searchsorted(cum, u, side="right")), k.size - 1)]))
    assert [int(x) for x in got] == want


def test_tensor_scale_and_cutoff(nb):
    a = nb.GpuSparseVector.from_entries(3, [1, 6, 1], [0.5, 0.5j, 0.25])  # duplicates add
    b = nb.GpuSparseVector.from_entries(2, [2, 3], [0.6, -0.8])
    ka, va = a.entries()
    assert list(ka) == [1, 6] and abs(va[0] - 0.75) < TOL
    t = a.tensor(b)
    assert t.num_qubits() == 5
    want = np.kron(b.to_vector(), a.to_vector())  # a on the low qubits
    assert np.abs(t.to_vector() - want).max() < TOL
    c = t.clone()
    c.scale(0.0)
    assert c.num_entries() == 0
    d = nb.GpuSparseVector.from_entries(4, [0, 1, 2], [1e-9, 0.6, 0.8]).with_cutoff(1e-6)
    assert sorted(int(x) for x in d.entries()[0]) == [1, 2]
    assert abs(d.amplitude(2) - 0.8) < TOL and d.amplitude(0) == 0


def test_errors(nb):
    with pytest.raises(nb.SimError):
        nb.GpuSparseVector(1025)  # registers of 1..1024 qubits
    s = nb.GpuSparseVector(4)
    with pytest.raises(nb.SimError):
        s.expectation(nb.Pauli(5, 0, 1, 0))
    with pytest.raises(nb.SimError):
        s.project(nb.Pauli(4, 1, 1, 0), False)  # XZ is not Hermitian
    with pytest.raises(nb.SimError) as e:
        s.run(nb.Circuit.parse("QUBITS 4\nH 0\n"), nb.StdRng(0))
        s.scale(0.0)
        s.sample(nb.StdRng(0), 3)
    assert e.value.kind == "ZeroState"


def poly_run_text(n, rng):
    """|+>^n, then phase polynomials over the whole register (20..44 terms of
    1..3 parities, half of them single bits, half multi-bit masks; 3- and 5-bit
    phases) interleaved with Toffoli and CNOT gates: one run of one-to-one ops."""
    lines = [f"QUBITS {n}"] + [f"H {q}" for q in range(n)]
    for _ in range(6):
        terms = []
        for _ in range(int(rng.integers(20, 45))):
            masks = [int(rng.integers(1, 1 << n)) if rng.random() < 0.5 else 1 << int(rng.integers(n))
                     for _ in range(int(rng.integers(1, 4)))]
            terms.append(f"{int(rng.integers(1, 32))}:" + ",".join(map(str, masks)))
        bits = int(rng.choice([3, 5]))
        lines.append(f"DIAG({bits};{int(rng.integers(1 << bits))};" + ";".join(terms) + ") "
                     + " ".join(map(str, range(n))))
        a, b, c = (int(v) for v in rng.choice(n, 3, replace=False))
        lines.append(f"CCX {a} {b} {c}")
        lines.append(f"CX {b} {c}")
    return "\n".join(lines) + "\n"


def test_phase_polynomials_in_a_run_match_the_dense_vector(nb, oracle):
    """Phase polynomials inside a run (the warp-shared term loads): single-bit and
    multi-bit parities, more than 32 terms, against the dense FP64 oracle."""
    rng = np.random.default_rng(21)
    for trial in range(4):
        n = 10 + trial
        text = poly_run_text(n, rng)
        s = nb.GpuSparseVector(n)
        s.run(nb.Circuit.parse(text), nb.StdRng(0))
        v = oracle.StateVector(n)
        v.run(oracle.Circuit(text), oracle.StdRng(0))
        assert s.num_entries() == 1 << n
        assert np.abs(s.to_vector() - v.to_vector()).max() < TOL, trial
