"""Seeded random Clifford circuits for the frame-sampler tests: every gate kind
the sampler distinguishes (named Cliffords, Paulis, Clifford phase gates,
diagonal and monomial Cliffords), Z/X/Y and product measurements, resets,
every noise channel and detectors / observables."""
from __future__ import annotations

import random

ONE = ["H", "S", "S_DAG", "SQRT_X", "SQRT_X_DAG", "SQRT_Y", "SQRT_Y_DAG", "X", "Y", "Z", "I",
       "PHASE(1,2)", "PHASE(2,2)", "PHASE(4,3)"]
# CPHASE(1,1) is CZ; the DIAG is S x S x CZ on its two variables; the MONOMIAL
# is CX with a shift and an S-type phase (all Clifford)
TWO = ["CX", "CY", "CZ", "SWAP", "CPHASE(1,1)", "CPHASE(2,2)", "DIAG(2;0;1:1;1:2;2:3)",
       "MONOMIAL(1,3;1;2;0;1:1;0,0,0)"]
NOISE1 = ["X_ERROR(0.1)", "Y_ERROR(0.05)", "Z_ERROR(0.2)", "DEPOLARIZE1(0.15)", "PAULI_CHANNEL_1(0.05,0.1,0.15)",
          "X_ERROR(0.3)", "Z_ERROR(0)"]


def random_clifford_text(r: random.Random, n: int, ops: int, noise: bool = True) -> str:
    lines = [f"QUBITS {n}"]
    m = 0
    for _ in range(ops):
        u = r.random()
        if u < 0.35:
            lines.append(f"{r.choice(ONE)} {r.randrange(n)}")
        elif u < 0.6 and n >= 2:
            a, b = r.sample(range(n), 2)
            lines.append(f"{r.choice(TWO)} {a} {b}")
        elif u < 0.72:
            lines.append(f"{r.choice(['M', 'MX', 'MY'])} {r.randrange(n)}")
            m += 1
        elif u < 0.78:
            qs = r.sample(range(n), r.randint(1, min(n, 4)))
            lines.append("MPP " + r.choice(["", "-"]) + "*".join(f"{r.choice('XYZ')}{q}" for q in qs))
            m += 1
        elif u < 0.83:
            lines.append(f"R {r.randrange(n)}")
        elif noise and u < 0.93:
            lines.append(f"{r.choice(NOISE1)} {r.randrange(n)}")
        elif noise and n >= 2:
            a, b = r.sample(range(n), 2)
            lines.append(f"DEPOLARIZE2({r.choice([0.01, 0.3])}) {a} {b}")
        if m and r.random() < 0.12:
            ks = sorted(r.sample(range(1, m + 1), r.randint(1, min(m, 3))))
            lines.append("DETECTOR " + " ".join(f"rec[-{k}]" for k in ks))
        if m and r.random() < 0.04:
            lines.append(f"OBSERVABLE_INCLUDE({r.randint(0, 1)}) rec[-{r.randint(1, m)}]")
    return "\n".join(lines) + "\n"


def batch_seeds(rng, shots: int) -> list[int]:
    """One next_u64 per batch of 16384 shots, in order (frame.rs:72-74)."""
    return [rng.next_u64() for _ in range((shots + (1 << 14) - 1) >> 14)]
