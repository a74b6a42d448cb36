"""Wide gates on the plain path: dense matrices on 6..13 qubits and monomial
tables on more than 10 qubits, which the reference applies through the same
fiber kernel as any other gate (src/state/vector.rs:67-93 and :130-137;
12-qubit Clifford unitaries reach it through src/clifford/mod.rs:317-318).

Dense gates are checked against the oracle's apply_matrix (every amplitude
within 1e-12 for complex128), monomial tables against a numpy application of
the same table (indices exact, values within 1e-12).
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _random_unitary(k: int, rng: np.random.Generator) -> np.ndarray:
    d = 1 << k
    z = rng.normal(size=(d, d)) + 1j * rng.normal(size=(d, d))
    q, r = np.linalg.qr(z)
    return q * (np.diag(r) / np.abs(np.diag(r)))


def _random_state(n: int, rng: np.random.Generator) -> np.ndarray:
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return v / np.linalg.norm(v)


def _apply_table(v: np.ndarray, n: int, qubits, image, phase) -> np.ndarray:
    """numpy: U|x> = phase[x] |image[x]> on the local index of `qubits`."""
    idx = np.arange(1 << n, dtype=np.int64)
    loc = np.zeros(1 << n, dtype=np.int64)
    for j, q in enumerate(qubits):
        loc |= ((idx >> q) & 1) << j
    rest = idx.copy()
    for q in qubits:
        rest &= ~(1 << q)
    img = np.asarray(image, dtype=np.int64)[loc]
    dst = rest.copy()
    for j, q in enumerate(qubits):
        dst |= ((img >> j) & 1) << q
    out = np.zeros_like(v)
    out[dst] = np.asarray(phase)[loc] * v
    return out


@pytest.mark.parametrize("k", [6, 7, 8, 9, 10, 11, 12])
def test_dense_gate_on_k_qubits_matches_oracle(nb, oracle, k):
    n = 15
    rng = np.random.default_rng(100 + k)
    u = _random_unitary(k, rng)
    qubits = [int(q) for q in rng.permutation(n)[:k]]
    v = _random_state(n, rng)
    g = nb.GpuStateVector.from_amplitudes(v)
    g.apply_matrix(u, qubits)
    o = oracle.StateVector.from_amplitudes(v)
    o.apply_matrix(u, qubits)
    assert np.abs(g.to_vector() - o.to_vector()).max() < TOL


def test_dense_gate_through_the_gate_view_and_complex64(nb, oracle):
    """Gate::Unitary on 8 qubits through apply_gate (lowering + check_qubits), and
    the same matrix on a complex64 register (within single precision)."""
    n, k = 14, 8
    rng = np.random.default_rng(7)
    u = _random_unitary(k, rng)
    qubits = [13, 0, 5, 2, 9, 11, 1, 7]
    v = _random_state(n, rng)
    o = oracle.StateVector.from_amplitudes(v)
    o.apply_matrix(u, qubits)
    g = nb.GpuStateVector.from_amplitudes(v)
    g.apply_gate(nb.Gate.unitary(u), qubits)
    assert np.abs(g.to_vector() - o.to_vector()).max() < TOL
    f = nb.GpuStateVector.from_amplitudes(v, nb.C64)
    f.apply_gate(nb.Gate.unitary(u), qubits)
    assert np.abs(f.to_vector() - o.to_vector()).max() < 2e-6
    with pytest.raises(nb.SimError) as e:
        g.apply_gate(nb.Gate.unitary(u), qubits[:7])
    assert e.value.kind == "Arity"


def test_thirteen_qubit_gate_on_the_whole_register(nb, oracle):
    """k = n = 13: a single fiber, a 8192 x 8192 matrix (1 GiB of complex128)."""
    n = 13
    rng = np.random.default_rng(13)
    # a sparse unitary (a permutation with phases, like a Clifford's dense view) keeps the host side quick
    perm = rng.permutation(1 << n)
    ph = np.exp(2j * np.pi * rng.integers(0, 8, size=1 << n) / 8)
    u = np.zeros((1 << n, 1 << n), dtype=np.complex128)
    u[perm, np.arange(1 << n)] = ph
    v = _random_state(n, rng)
    qubits = [int(q) for q in rng.permutation(n)]
    g = nb.GpuStateVector.from_amplitudes(v)
    g.apply_matrix(u, qubits)
    want = _apply_table(v, n, qubits, perm, ph)
    assert np.abs(g.to_vector() - want).max() < TOL


@pytest.mark.parametrize("k", [11, 12, 14])
def test_monomial_table_on_k_qubits(nb, k):
    n = 16
    rng = np.random.default_rng(200 + k)
    image = rng.permutation(1 << k)
    phase = np.exp(2j * np.pi * rng.integers(0, 8, size=1 << k) / 8)
    phase[rng.random(1 << k) < 0.3] = 1.0
    qubits = [int(q) for q in rng.permutation(n)[:k]]
    v = _random_state(n, rng)
    g = nb.GpuStateVector.from_amplitudes(v)
    g.apply_monomial(qubits, image, phase)
    want = _apply_table(v, n, qubits, image, phase)
    got = g.to_vector()
    assert np.array_equal(np.nonzero(got)[0], np.nonzero(want)[0])
    assert np.abs(got - want).max() < TOL
    f = nb.GpuStateVector.from_amplitudes(v, nb.C64)
    f.apply_monomial(qubits, image, phase)
    assert np.abs(f.to_vector() - want).max() < 2e-6


def test_diagonal_table_on_twelve_qubits(nb):
    n, k = 15, 12
    rng = np.random.default_rng(5)
    phase = np.exp(2j * np.pi * rng.random(1 << k))
    qubits = [int(q) for q in rng.permutation(n)[:k]]
    v = _random_state(n, rng)
    g = nb.GpuStateVector.from_amplitudes(v)
    g.apply_monomial(qubits, np.arange(1 << k), phase)
    assert np.abs(g.to_vector() - _apply_table(v, n, qubits, np.arange(1 << k), phase)).max() < TOL


def test_wide_gate_limits(nb):
    """Dense gates on more than 13 qubits are refused before the matrix is read."""
    import ctypes as C

    g = nb.GpuStateVector(15)
    q = (C.c_uint32 * 14)(*range(14))
    dummy = (C.c_double * 2)()
    st = nb.lib().ncsim_sv_apply_matrix(g._h, q, 14, dummy)
    assert st == 1 and "13" in nb.lib().ncsim_last_error().decode()
