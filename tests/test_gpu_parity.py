"""Parity of the CUDA engine with the CPU oracle (the restatement of ncsim's
``StateVector<C64>``), through the C ABI.

Tolerances: complex128 states within 1e-12 per amplitude (the drop-in
contract); complex64 states within 2e-6 per amplitude of unit-norm states;
indices (sampling, monomial images, nonzero sets) bit-exact; measurement
records identical for the same seeded StdRng.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

import numpy_sim

pytestmark = pytest.mark.gpu

TOL = 1e-12
TOL_C64 = 2e-6


def rand_state(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return v / np.linalg.norm(v)


def pair(nb, oracle, n, seed, precision=0):
    v = rand_state(n, seed)
    g = nb.GpuStateVector.from_amplitudes(v, precision)
    o = oracle.StateVector.from_amplitudes(v)
    return g, o


def maxerr(g, o):
    return float(np.abs(g.to_vector() - o.to_vector()).max())


def test_golden_circuits_on_device(nb, golden):
    for fx in golden["circuits"]:
        n = fx["n"]
        s = nb.GpuStateVector(n)
        s.run(nb.Circuit.parse(fx["text"]), nb.StdRng(0))
        want = np.zeros(1 << n, dtype=complex)
        want[fx["indices"]] = [complex(a, b) for a, b in fx["amplitudes"]]
        assert np.abs(s.to_vector() - want).max() < TOL, fx["name"]


ONE_Q = ["I", "X", "Y", "Z", "H", "S", "S_DAG", "SQRT_X", "SQRT_X_DAG", "SQRT_Y", "SQRT_Y_DAG", "T", "T_DAG",
         "PHASE(3,4)", "PHASE(5,7)", "RX(0.3)", "RY(1.1)", "RZ(2.2)"]
TWO_Q = ["CX", "CY", "CZ", "SWAP", "CS", "CS_DAG", "CPHASE(1,3)"]
THREE_Q = ["CCZ", "CCX"]


@pytest.mark.parametrize("precision", [0, 1])
def test_every_named_gate_on_every_placement(nb, oracle, precision):
    n = 12
    g, o = pair(nb, oracle, n, 1, precision)
    placements = {1: [[q] for q in range(n)],
                  2: [[0, 1], [1, 0], [0, 11], [11, 0], [5, 6], [3, 9], [10, 2], [4, 1]],
                  3: [[0, 1, 2], [2, 1, 0], [0, 5, 11], [11, 6, 0], [3, 9, 7], [1, 10, 4]]}
    tol = TOL if precision == 0 else TOL_C64 * 4
    for names, k in ((ONE_Q, 1), (TWO_Q, 2), (THREE_Q, 3)):
        for name in names:
            gate = nb.Gate.parse(name)
            for qs in placements[k]:
                g.apply_gate(gate, qs)
                o.apply_gate_text(f"{name} " + " ".join(map(str, qs)))
    assert maxerr(g, o) < tol


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("k", [1, 2, 3, 4, 5])
def test_dense_matrices_against_oracle(nb, oracle, k, precision):
    rng = np.random.default_rng(k)
    n = 12
    g, o = pair(nb, oracle, n, 2, precision)
    for trial in range(6):
        qs = [int(q) for q in rng.permutation(n)[:k]]
        if trial == 0:
            qs = list(range(k))  # all low qubits
        if trial == 1:
            qs = list(range(n - k, n))[::-1]  # all high, reversed
        m = rng.normal(size=(1 << k, 1 << k)) + 1j * rng.normal(size=(1 << k, 1 << k))
        m /= np.abs(m).sum(axis=1, keepdims=True)
        g.apply_matrix(m, qs)
        o.apply_matrix(m, qs)
    assert maxerr(g, o) < (TOL if precision == 0 else TOL_C64)


def test_monomial_tables_and_shapes(nb, oracle):
    rng = np.random.default_rng(3)
    n = 13
    g, o = pair(nb, oracle, n, 3)
    for k in (1, 2, 3, 5, 8, 10):
        for trial in range(3):
            qs = [int(q) for q in rng.permutation(n)[:k]]
            d = 1 << k
            img = rng.permutation(d)
            ph = np.exp(2j * np.pi * rng.integers(0, 8, size=d) / 8)
            if trial == 1:
                img = np.arange(d)  # diagonal table
            m = np.zeros((d, d), dtype=complex)
            m[img, np.arange(d)] = ph
            g.apply_monomial(qs, img, ph)
            if k <= 5:
                o.apply_matrix(m, qs)
            else:
                full = numpy_sim.NumpyState(n)
                full.v = o.to_vector()
                full.apply(m, qs)
                o.set_amplitudes(full.v)
    assert maxerr(g, o) < TOL


def test_monomial_and_diagonal_gates_from_text(nb, oracle):
    text = oracle.reversible_circuit_text(14, 120, 11)
    g = nb.GpuStateVector(14)
    g.run(nb.Circuit.parse(text), nb.StdRng(0))
    o = oracle.StateVector(14)
    o.run(oracle.Circuit(text), oracle.StdRng(0))
    a, b = g.to_vector(), o.to_vector()
    assert np.array_equal(np.flatnonzero(a), np.flatnonzero(b))
    assert np.abs(a - b).max() < TOL


@pytest.mark.parametrize("bits,scalar,precision", [(3, (0, 0, 0), 0), (5, (1, 3, 2), 0), (8, (0, 1, 3), 0), (1, (0, 0, 0), 1),
                                                   (3, (2, 1, 2), 1), (12, (0, 0, 0), 0), (12, (-2, 5, 3), 0)])
def test_phase_polynomial_from_the_bit_index(nb, oracle, bits, scalar, precision):
    """Exponents of at most 8 bits take the bit-sliced kernel (a warp per
    1024 amplitudes); wider ones the per-amplitude form."""
    n = 12
    rng = np.random.default_rng(bits)
    g, o = pair(nb, oracle, n, 4, precision)
    qs = [int(q) for q in rng.permutation(n)]
    terms = []
    for _ in range(25):
        deg = int(rng.integers(1, 4))
        pars = [int(rng.integers(1, 1 << n)) for _ in range(deg)]
        terms.append((int(rng.integers(1, 1 << bits)), pars))
    const = int(rng.integers(0, 1 << bits))
    g.apply_phasepoly(qs, bits, const, terms, scalar)
    # the same function, evaluated on the host
    v = o.to_vector()
    idx = np.arange(1 << n, dtype=np.int64)
    x = np.zeros_like(idx)
    for j, q in enumerate(qs):
        x |= ((idx >> q) & 1) << j
    f = np.full(idx.shape, const, dtype=np.int64)
    for c, pars in terms:
        prod = np.ones_like(idx)
        for p in pars:
            prod &= np.array([bin(int(t) & p).count("1") & 1 for t in x])
        f = f + c * prod
    f %= 1 << bits
    s2, sp, sb = scalar
    factor = (math.sqrt(2) ** s2) * np.exp(2j * np.pi * sp / (1 << sb)) * np.exp(2j * np.pi * f / (1 << bits))
    tol = TOL * abs(math.sqrt(2) ** s2) if precision == 0 else TOL_C64 * max(1.0, math.sqrt(2) ** s2)
    assert np.abs(g.to_vector() - v * factor).max() < tol


def test_paulis_readouts_and_projections(nb, oracle):
    rng = np.random.default_rng(5)
    n = 14
    g, o = pair(nb, oracle, n, 5)
    g2, o2 = pair(nb, oracle, n, 6)
    for trial in range(12):
        x = int(rng.integers(0, 1 << n)) if trial % 4 else 0
        z = int(rng.integers(0, 1 << n))
        ph = bin(x & z).count("1") % 4
        if trial % 3 == 0:
            ph = (ph + 2) % 4
        p = nb.Pauli(n, x, z, ph)
        assert abs(g.expectation(p) - o.expectation_raw(x, z, ph)) < TOL
        e, nn = g.measure_stats(p)
        assert abs(e - o.expectation_raw(x, z, ph)) < TOL and abs(nn - o.norm_sq().real) < TOL
        q = nb.Pauli(n, x, z, (ph + 1) % 4)  # non-Hermitian: apply only
        g.apply_pauli(q)
        o.apply_pauli_raw(x, z, (ph + 1) % 4)
        gc, oc = g.clone(), o.clone()
        b = bool(trial % 2)
        w1, w2 = gc.project(p, b), oc.project_raw(x, z, ph, b)
        assert abs(w1 - w2) < TOL
        assert maxerr(gc, oc) < TOL
    assert maxerr(g, o) < TOL
    assert abs(g.inner(g2) - o.inner(o2)) < TOL
    assert abs(g.norm_sq() - o.norm_sq()) < TOL
    g.scale(0.3 - 0.7j)
    o.scale(0.3 - 0.7j)
    assert maxerr(g, o) < TOL
    g.normalize()
    o.normalize()
    assert maxerr(g, o) < TOL
    assert abs(g.probability(77) - abs(o.to_vector()[77]) ** 2 / o.norm_sq().real) < TOL
    terms = [(0.5, nb.Pauli(n, 3, 0, 0)), (-1.25j, nb.Pauli(n, 0, 5, 0)), (2.0, nb.Pauli(n, 8, 8, 1))]
    want = sum(c * o.expectation_raw(p.x, p.z, p.phase) for c, p in terms)
    assert abs(g.expectation_sum(terms) - want) < TOL
    with pytest.raises(nb.SimError) as ei:
        g.project(nb.Pauli(n, 1, 1, 0), False)  # XZ with phase 0 is not Hermitian
    assert ei.value.kind == "Invalid"


def test_sampling_matches_oracle_and_the_born_rule(nb, oracle):
    """src/state/vector.rs:767-800 on the device, and shot-for-shot against the oracle."""
    n = 14
    i = np.arange(1 << n)
    amps = np.where(i % 4099 == 7, 3.0, 0.01 * (i % 13)).astype(complex)
    g = nb.GpuStateVector.from_amplitudes(amps)
    o = oracle.StateVector.from_amplitudes(amps)
    u = np.random.default_rng(9).random(200_000)
    sg, so = g.sample_uniforms(u), o.sample_uniforms(u)
    assert np.array_equal(sg, so)
    s = g.sample(nb.StdRng(2), 200_000).astype(np.int64)
    assert np.array_equal(s, o.sample(oracle.StdRng(2), 200_000).astype(np.int64))
    assert np.all((s % 13 != 0) | (s % 4099 == 7))
    total = np.sum(np.abs(amps) ** 2)
    counts = np.bincount(s, minlength=1 << n)
    for k in range(7, 1 << n, 4099):
        p = abs(amps[k]) ** 2 / total
        assert abs(counts[k] / s.size - p) < 6 * math.sqrt(p * (1 - p) / s.size)


def test_random_layers_c0_config(nb, oracle):
    """n = 20, depth 40, seed 1: amplitudes, <Z0 Z1>, <X0 X5 Y9>, 4096 samples, 64 amplitudes."""
    n = 20
    cg = nb.Circuit.random_layers(n, 40, 1)
    text = oracle.random_circuit_text(n, 40, 1)
    g = nb.GpuStateVector(n)
    o = oracle.StateVector(n)
    g.run(cg, nb.StdRng(1))
    o.run(oracle.Circuit(text), oracle.StdRng(1))
    assert maxerr(g, o) < TOL
    for ptxt in ("Z0*Z1", "X0*X5*Y9"):
        assert abs(g.expectation(nb.Pauli.from_string(n, ptxt)) - o.expectation(ptxt)) < TOL
    rg2, ro2 = nb.StdRng(99), oracle.StdRng(99)
    assert np.array_equal(g.sample(rg2, 4096), o.sample(ro2, 4096))
    idx = [rg2.gen_range(0, 1 << n) for _ in range(64)]
    assert idx == [ro2.gen_range(0, 1 << n) for _ in range(64)]
    assert np.abs(g.amplitudes_at(idx) - o.to_vector()[idx]).max() < TOL


def test_random_layers_with_measurements(nb, oracle):
    """The C1 family at n = 24 (records on the final 4 qubits identical, amplitudes within 1e-12)."""
    n = 24
    text = oracle.random_circuit_text(n, 20, 1, 0.0, n - 4, n)
    g = nb.GpuStateVector(n)
    o = oracle.StateVector(n)
    rec_g = g.run(nb.Circuit.parse(text), nb.StdRng(5))
    rec_o = o.run(oracle.Circuit(text), oracle.StdRng(5))
    assert rec_g == rec_o and len(rec_g) == 4
    assert maxerr(g, o) < TOL


def test_gate_runs_replayed_as_graphs(nb, oracle):
    """Runs of gates are captured as CUDA graphs on the second run of a circuit on
    a state and replayed by later runs; measurements in between stay direct.  The
    register after each run, and the records, match the oracle; a run with the
    launch profiler on (direct launches) gives the same register."""
    n = 14
    text = oracle.random_circuit_text(n, 6, 9) + "M 3\n" + oracle.random_circuit_text(n, 4, 10).split("\n", 1)[1]
    g = nb.GpuStateVector(n)
    o = oracle.StateVector(n)
    rg, ro = nb.StdRng(5), oracle.StdRng(5)
    c, oc = nb.Circuit.parse(text), oracle.Circuit(text)
    for _ in range(3):
        assert g.run(c, rg) == o.run(oc, ro)
        assert maxerr(g, o) < TOL
    p = nb.GpuStateVector(n)
    p.profile(True)
    p.run(c, nb.StdRng(5))
    q = nb.GpuStateVector(n)
    q.run(c, nb.StdRng(5))
    assert np.abs(p.to_vector() - q.to_vector()).max() < TOL
    assert p.profile_read()  # the profiled run launched kernel by kernel


def test_noisy_trajectories_match_oracle(nb, oracle):
    """The batched family's per-trajectory semantics on the plain path (complex128)."""
    for t in range(3):
        seed = 1 + t
        n_o, z0_o, rec_o = oracle.trajectory(seed, 12, 5, 8, 0.05)
        rng = nb.StdRng(seed)
        n = 12 + rng.gen_range(0, 5)
        assert n == n_o
        c = nb.Circuit.random_layers_from(rng, n, 8, 0.05, 0, 0)
        s = nb.GpuStateVector(n)
        s.run(c, rng)
        e = s.expectation(nb.Pauli(n, 0, 1, 0)).real / s.norm_sq().real
        assert abs(e - z0_o) < TOL
        m = nb.Circuit.parse(f"QUBITS {n}\n" + "".join(f"M {q}\n" for q in range(n)))
        assert s.run(m, rng) == rec_o


def test_reversible_family_dense(nb, oracle):
    text = oracle.reversible_circuit_text(20, 400, 2)
    g = nb.GpuStateVector(20)
    g.run(nb.Circuit.parse(text), nb.StdRng(0))
    idx, amp = oracle.sparse_run(text)
    a = g.to_vector()
    assert np.array_equal(np.flatnonzero(a), idx.astype(np.int64))
    assert np.abs(a[idx.astype(np.int64)] - amp).max() < TOL


@pytest.mark.parametrize("precision", [0, 1])
def test_reversible_family_on_a_dense_state(nb, oracle, precision):
    """Every amplitude nonzero: the 40-term diagonals and the 8-qubit
    monomials of the reversible family act on all 2^n entries (the bit-sliced
    phase-polynomial kernel and the tiled permutation kernel)."""
    n = 16
    text = oracle.reversible_circuit_text(n, 150, 9)
    g, o = pair(nb, oracle, n, 12, precision)
    g.run(nb.Circuit.parse(text), nb.StdRng(0))
    o.run(oracle.Circuit(text), oracle.StdRng(0))
    tol = TOL if precision == 0 else TOL_C64 * 2 ** (-n / 2) * 16
    assert maxerr(g, o) < tol


def test_complex64_storage_plain_path(nb, oracle):
    n = 16
    text = oracle.random_circuit_text(n, 10, 4)
    g = nb.GpuStateVector(n, nb.C64)
    o = oracle.StateVector(n)
    g.run(nb.Circuit.parse(text), nb.StdRng(0))
    o.run(oracle.Circuit(text), oracle.StdRng(0))
    a, b = g.to_vector(), o.to_vector()
    assert np.abs(a - b).max() < TOL_C64 * 2 ** (-n / 2) * 64
    assert abs(g.norm_sq().real - 1) < 1e-5


def test_kron_clone_and_basis_states(nb, oracle):
    a, oa = pair(nb, oracle, 5, 7)
    b, ob = pair(nb, oracle, 4, 8)
    k = a.tensor(b)
    assert k.n == 9
    assert np.abs(k.to_vector() - oa.kron(ob).to_vector()).max() < TOL
    c = k.clone()
    c.apply_gate(nb.Gate.parse("H"), [3])
    assert np.abs(k.to_vector() - oa.kron(ob).to_vector()).max() < TOL
    s = nb.GpuStateVector.basis_state(6, 37)
    assert s.amplitude(37) == 1 and s.norm_sq() == 1
    p = nb.GpuStateVector.plus_state(7)
    assert np.allclose(p.to_vector(), 2 ** -3.5, atol=0, rtol=1e-15)


def test_argument_errors_on_device(nb):
    s = nb.GpuStateVector(6)
    h = nb.Gate.parse("H")
    # check_qubits runs before the arity check (vector.rs:365-372)
    for qs, kind in (([6], "QubitOutOfRange"), ([1, 1], "DuplicateQubit"), ([1, 2], "Arity"), ([], "Arity")):
        with pytest.raises(nb.SimError) as e:
            s.apply_gate(h, qs)
        assert e.value.kind == kind
    with pytest.raises(nb.SimError) as e:
        s.apply_gate(nb.Gate.parse("CX"), [2, 2])
    assert e.value.kind == "DuplicateQubit"
    # the variants' fields cross the ABI (error.rs:17-33)
    with pytest.raises(nb.SimError) as e:
        s.apply_gate(nb.Gate.parse("CCZ"), [0, 9, 1])
    assert e.value.kind == "QubitOutOfRange" and e.value.fields == {"qubit": 9, "num_qubits": 6}
    with pytest.raises(nb.SimError) as e:
        s.apply_gate(nb.Gate.parse("CZ"), [3, 4, 3])
    assert e.value.fields == {"qubit": 3}
    with pytest.raises(nb.SimError) as e:
        s.apply_gate(nb.Gate.parse("CCZ"), [0, 1])
    assert e.value.fields == {"gate": "CCZ", "expected": 3, "got": 2}
    with pytest.raises(nb.SimError) as e:
        s.apply_matrix(np.eye(4), [0, 7])
    assert e.value.fields == {"qubit": 7, "num_qubits": 6}
    with pytest.raises(nb.SimError) as e:
        s.run(nb.Circuit.parse("QUBITS 5\nH 0\n"), nb.StdRng(0))
    assert e.value.kind == "Invalid"
    s.project(nb.Pauli(6, 0, 1, 0), True)  # |0..0> projected on Z0 = -1 vanishes
    with pytest.raises(nb.SimError) as e:
        s.sample(nb.StdRng(0), 4)
    assert e.value.kind == "ZeroState"
    with pytest.raises(nb.SimError) as e:
        s.normalize()
    assert e.value.kind == "ZeroState"


@pytest.mark.slow
def test_reversible_family_full_size_against_sparse_oracle(nb, oracle):
    """n = 31 complex128 (32 GiB), 2000 permutation/diagonal gates: the 2^16
    nonzero entries bit-exact in index and within 1e-12 in value, and the
    rest of the register empty (its norm equals theirs)."""
    n = 31
    info = nb.device_info()
    if info["free_bytes"] < (16 << n) + (4 << 30):
        pytest.skip("needs 36 GiB of free device memory")
    c = nb.Circuit.reversible(n, 2000, 1)
    g = nb.GpuStateVector(n)
    g.run(c, nb.StdRng(0))
    idx, amp = oracle.sparse_run(c.to_text())
    assert idx.size == 1 << 16
    got = g.amplitudes_at(idx)
    assert np.abs(got - amp).max() < TOL
    assert abs(g.norm_sq().real - np.sum(np.abs(amp) ** 2)) < 1e-12
