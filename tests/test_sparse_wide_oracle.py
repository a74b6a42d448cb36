"""The oracle's sparse restatement on registers of any width (Bits keys), pinned
before the wide GPU sparse form is checked against it.

- Against the dense oracle on 12-qubit circuits from the wide generator:
  records identical, amplitudes within 1e-12 (the same gate views and draw
  order, sparse.rs:131-231 and mod.rs:113-183).
- The reference's published SparseVector workload (examples/bench.rs:245-262)
  as a known answer: every entry is the classical ripple image of its input,
  in the input order (H's leave the entries sorted, the ripple moves them in
  place), with amplitude 2^-inputs/2.
- Sampling walks the cumulative weights in entry order (sparse.rs:407-424),
  restated here in Python from the same StdRng draws.
"""
from __future__ import annotations

import bisect

import numpy as np
import pytest

from tests.wide_cases import random_wide_text, ripple_image, ripple_text


@pytest.fixture(scope="module")
def oracle():
    from oracle import oracle as O

    O.build()
    return O


@pytest.mark.parametrize("seed", range(6))
def test_wide_restatement_matches_the_dense_oracle(oracle, seed):
    n = 12
    text = random_wide_text(n, 60, seed)
    w = oracle.WideSparse(text, 100 + seed)
    d = oracle.StateVector(n)
    rec = d.run(oracle.Circuit(text), oracle.StdRng(100 + seed))
    assert w.record == rec
    keys, amps = w.entries()
    v = np.zeros(1 << n, dtype=np.complex128)
    for k, a in zip(keys, amps):
        v[k] = a
    assert np.abs(v - d.to_vector()).max() < 1e-12
    assert len(set(keys)) == len(keys)
    assert all(a != 0 for a in amps)


def test_published_ripple_is_a_permutation_of_the_inputs(oracle):
    n, inputs = 200, 10
    w = oracle.WideSparse(ripple_text(n, inputs), 1)
    keys, amps = w.entries()
    assert keys == [ripple_image(x, n) for x in range(1 << inputs)]
    assert np.allclose(amps, 2.0 ** (-inputs / 2), atol=1e-15, rtol=0)
    # <Z0 Z(n-1)> from the entries
    want = sum(abs(a) ** 2 * (-1) ** (((k >> 0) & 1) ^ ((k >> (n - 1)) & 1)) for k, a in zip(keys, amps))
    assert abs(w.expectation(f"Z0*Z{n - 1}").real - want) < 1e-12


def test_sampling_follows_the_entry_order(oracle):
    n = 130
    w = oracle.WideSparse(ripple_text(n, 6), 1)
    keys, amps = w.entries()
    cum = np.cumsum(amps.real ** 2 + amps.imag ** 2)
    rng = oracle.StdRng(77)
    want = []
    for _ in range(300):
        u = rng.gen_f64() * cum[-1]
        want.append(keys[min(bisect.bisect_right(cum, u), len(keys) - 1)])
    assert w.sample(77, 300) == want
