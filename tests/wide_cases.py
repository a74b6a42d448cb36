"""Circuits on registers wider than 64 qubits for the sparse form's tests.

ripple_text: the reference's published SparseVector workload
(examples/bench.rs:245-262): H on the first `inputs` qubits of an n-qubit
register, then for q in 0..n-2 a CCX on (q, q+1, q+2) and a CX on (q, q+2).
ripple_image: the same gates applied classically to one basis index.
random_wide_text: seeded random circuits mixing dense, permutation, diagonal
and Pauli gates with measurements, resets and Pauli noise.
"""
from __future__ import annotations

import random


def ripple_text(n: int = 1000, inputs: int = 10) -> str:
    lines = [f"QUBITS {n}"] + [f"H {q}" for q in range(inputs)]
    for q in range(n - 2):
        lines.append(f"CCX {q} {q + 1} {q + 2}")
        lines.append(f"CX {q} {q + 2}")
    return "\n".join(lines) + "\n"


def ripple_image(x: int, n: int) -> int:
    for q in range(n - 2):
        if (x >> q) & 1 and (x >> (q + 1)) & 1:
            x ^= 1 << (q + 2)
        if (x >> q) & 1:
            x ^= 1 << (q + 2)
    return x


ONE_QUBIT = ["H", "SQRT_X", "S", "T", "X", "Y", "Z", "SQRT_Y", "T_DAG"]
TWO_QUBIT = ["CX", "CZ", "SWAP", "CS", "CY"]


def random_wide_text(n: int, gates: int, seed: int, dense_budget: int = 8, measure: bool = True,
                     noise: bool = True) -> str:
    """Gates on qubits spread over the whole register; at most `dense_budget`
    entry-doubling gates (H, SQRT_X, SQRT_Y, RX) so the state stays small."""
    r = random.Random(seed)
    lines = [f"QUBITS {n}"]
    dense = 0
    hot = r.sample(range(n), min(n, 12))  # most gates land on a few qubits, so they interact
    for _ in range(gates):
        qs = lambda k: r.sample(hot, k) if r.random() < 0.8 else r.sample(range(n), k)  # noqa: E731
        u = r.random()
        if u < 0.45:
            g = r.choice(ONE_QUBIT)
            if g in ("H", "SQRT_X", "SQRT_Y"):
                if dense >= dense_budget:
                    g = "T"
                else:
                    dense += 1
            lines.append(f"{g} {qs(1)[0]}")
        elif u < 0.5:
            if dense < dense_budget:
                dense += 1
                lines.append(f"RX({r.uniform(-3, 3):.6f}) {qs(1)[0]}")
            else:
                lines.append(f"RZ({r.uniform(-3, 3):.6f}) {qs(1)[0]}")
        elif u < 0.8:
            a, b = qs(2)
            lines.append(f"{r.choice(TWO_QUBIT)} {a} {b}")
        elif u < 0.88:
            a, b, c = qs(3)
            lines.append(f"{r.choice(['CCX', 'CCZ'])} {a} {b} {c}")
        elif u < 0.895:
            # diagonal phase polynomials: on 4 qubits (a monomial table) and on 11 (evaluated per entry)
            if r.random() < 0.5:
                lines.append(f"DIAG(3;1;1:1;3:2,4;5:1,2,8) {' '.join(map(str, qs(4)))}")
            else:
                lines.append(f"DIAG(4;3;5:1;3:6,1024;9:513,12,2) {' '.join(map(str, qs(11)))}")
        elif u < 0.93 and measure:
            lines.append(f"M {qs(1)[0]}")
        elif u < 0.95 and measure:
            lines.append(f"R {qs(1)[0]}")
        elif noise:
            lines.append(f"DEPOLARIZE1(0.2) {qs(1)[0]}")
    if measure:
        a, b = r.sample(hot, 2)
        lines.append(f"MPP X{a}*Z{b}")
    return "\n".join(lines) + "\n"
