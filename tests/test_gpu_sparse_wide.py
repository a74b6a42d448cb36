"""The sparse form on registers of 65..1024 qubits (multi-word keys) against the
oracle's restatement of sparse.rs with Bits keys.

- The reference's published workload (examples/bench.rs:245-262: n = 1000, H on
  10 qubits, a CCX/CX ripple of 1996 gates): entries in entry order, keys
  bit-exact and amplitudes within 1e-12, <Z0 Z999>, and Born samples shot for
  shot, through `run` (runs of one-to-one gates in one launch) and gate by gate.
- Seeded random circuits (dense, permutation, diagonal and Pauli gates,
  measurements, resets, Pauli noise) at n = 100, 300 and 1000: records
  identical, entries identical in order, expectations within 1e-12.
- from_entries (duplicates added, keys masked), tensor products past 64
  qubits, the W-word Pauli entry points and their argument checks.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from tests.wide_cases import random_wide_text, ripple_image, ripple_text

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nb():
    import ncsim_b200

    ncsim_b200.lib()
    return ncsim_b200


@pytest.fixture(scope="module")
def oracle():
    from oracle import oracle as O

    O.build()
    return O


def _bits_order(words):
    """Sort key of ncsim's Bits (Vec<u64>): word 0 first."""
    return lambda k: tuple((k >> (64 * i)) & 0xFFFFFFFFFFFFFFFF for i in range(words))


def _same_entries(g, o):
    gk, ga = g.entries()
    ok, oa = o.entries()
    assert list(gk) == list(ok)
    assert np.abs(np.asarray(ga) - np.asarray(oa)).max() < 1e-12


def test_published_ripple_at_1000_qubits(nb, oracle):
    n = 1000
    text = ripple_text(n, 10)
    o = oracle.WideSparse(text, 1)
    g = nb.GpuSparseVector(n)
    assert g.words == 16
    g.run(nb.Circuit.parse(text), nb.StdRng(1))
    _same_entries(g, o)
    keys, _ = g.entries()
    assert keys == [ripple_image(x, n) for x in range(1024)]
    p = nb.Pauli.from_string(n, "Z0*Z999")
    assert abs(g.expectation(p) - o.expectation("Z0*Z999")) < 1e-12
    assert g.sample(nb.StdRng(5), 2000) == o.sample(5, 2000)
    # gate by gate (no runs): the same entries
    h = nb.GpuSparseVector(n)
    for line in text.splitlines()[1:]:
        name, *qs = line.split()
        h.apply_gate(nb.Gate.parse(name), [int(q) for q in qs])
    _same_entries(h, o)


@pytest.mark.parametrize("n,seed", [(100, 1), (100, 2), (300, 3), (300, 4), (1000, 5), (1000, 6)])
def test_random_wide_circuits_match_the_oracle(nb, oracle, n, seed):
    text = random_wide_text(n, 150, seed)
    o = oracle.WideSparse(text, 40 + seed)
    g = nb.GpuSparseVector(n)
    rec = g.run(nb.Circuit.parse(text), nb.StdRng(40 + seed))
    assert rec == o.record
    _same_entries(g, o)
    keys, _ = g.entries()
    hot = sorted({int(t) for line in text.splitlines()[1:] for t in line.split()[1:] if t.isdigit()})[:6]
    for ptext in (f"Z{hot[0]}*Z{hot[1]}", f"X{hot[2]}", f"X{hot[0]}*Y{hot[3]}*Z{hot[4]}", f"Y{hot[5]}"):
        e = g.expectation(nb.Pauli.from_string(n, ptext))
        assert abs(e - o.expectation(ptext)) < 1e-12, ptext
    g.sort()
    assert g.entries()[0] == sorted(keys, key=_bits_order(g.words))


def test_from_entries_tensor_and_word_entry_points(nb):
    n = 300
    big = (1 << 299) | (1 << 170) | 5
    g = nb.GpuSparseVector.from_entries(n, [big, 7, big, (1 << 400) | 3], [0.5, 0.25j, 0.5, 1.0])
    keys, amps = g.entries()
    # masked to 300 qubits, duplicates added, sorted as Vec<u64> (word 0 first: big's word 0 is 5)
    assert keys == [3, big, 7]
    assert np.allclose(amps, [1.0, 1.0, 0.25j])
    assert abs(g.amplitude(big) - 1.0) < 1e-15 and g.amplitude(1 << 299) == 0
    # X on qubit 299 and Z on qubit 170 through the word entry points
    g.apply_pauli(nb.Pauli.from_string(n, "X299*Z170"))
    k2, a2 = g.entries()
    assert k2 == [3 | (1 << 299), big ^ (1 << 299), 7 | (1 << 299)]  # moved in place, order kept
    assert np.allclose(a2, [1.0, -1.0, 0.25j])
    w = g.project(nb.Pauli.from_string(n, "Z299"), False)  # keeps the entry without qubit 299
    assert abs(w - 1.0) < 1e-12 and g.entries()[0] == [big ^ (1 << 299)]
    # tensor past 64 qubits: a on the low qubits, b above them
    a = nb.GpuSparseVector(40)
    a.apply_gate(nb.Gate.parse("H"), [39])
    b = nb.GpuSparseVector(60)
    b.apply_gate(nb.Gate.parse("H"), [59])
    c = a.tensor(b)
    assert c.n == 100 and c.words == 4
    c.sort()
    ck, ca = c.entries()
    assert ck == [0, 1 << 99, 1 << 39, (1 << 99) | (1 << 39)]  # word 0 first
    assert np.allclose(ca, 0.5)
    # argument checks: word counts and bits outside the register
    s = nb.GpuSparseVector(200)
    x = (ctypes.c_uint64 * 3)()
    z = (ctypes.c_uint64 * 3)()
    assert nb.lib().ncsim_sparse_apply_pauli_words(s._h, x, z, 3, 0) == 8
    x4 = (ctypes.c_uint64 * 4)(0, 0, 0, 1 << 63)
    z4 = (ctypes.c_uint64 * 4)()
    assert nb.lib().ncsim_sparse_apply_pauli_words(s._h, x4, z4, 4, 0) == 8
