"""Generates the golden fixtures in this folder (test infrastructure).

The reference (Rust) cannot be built or run here, so the amplitudes come from
the independent numpy simulator (``tests/numpy_sim.py``), evaluated on the
reference's own test circuits (tests/backends.rs:18-33, src/state/vector.rs:582-583
and 637-643) and on small members of the seeded workload families.  The
ChaCha20 keystream vectors are RFC 8439, Appendix A.1, test vectors #1 and #2.

Run from the repository root: ``python tests/golden/make_golden.py``.
"""
from __future__ import annotations

import json
import os
import struct
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

import numpy_sim  # noqa: E402

CLIFFORD_T = """QUBITS 4
H 0 1 2 3
T 0
CX 0 1
CS 1 2
T_DAG 3
CZ 2 3
H 1
CCZ 0 1 2
SQRT_X 3
S 0
CX 3 0
H 2
T 2
"""

GHZ = "QUBITS 3\nH 0\nCX 0 1\nCX 1 2\n"

NON_CLIFFORD = "QUBITS 2\nH 0\nH 1\nT 0\nCS 0 1\nSQRT_X 1\nRZ(0.7) 0\n"

MISC = (
    "QUBITS 5\nH 0 1 2 3 4\nCY 0 1\nSWAP 1 3\nPHASE(3,4) 2\nCPHASE(5,3) 0 2\nRX(0.3) 1\nRY(1.1) 2\n"
    "SQRT_Y 3\nSQRT_Y_DAG 0\nSQRT_X_DAG 1\nCS 2 3\nCS_DAG 1 0\nY 2\nCCX 3 1 0\nT_DAG 1\nS_DAG 2\n"
    "X 4\nZ 3\nCCZ 4 0 2\nTOFFOLI 2 4 1\nCNOT 4 3\nI 0\n"
)


def chacha_vectors():
    k1 = "76b8e0ada0f13d90405d6ae55386bd28bdd219b8a08ded1aa836efcc8b770dc7da41597c5157488d7724e03fb8d84a376a43b8f41518a11cc387b669b2ee6586"
    k2 = "9f07e7be5551387a98ba977c732d080dcb0f29a048e3656912c6533e32ee7aed29b721769ce64e43d57133b074d839d531ed1f28510afb45ace10a1f4b794d6f"
    return [
        {"key": [0] * 8, "counter": 0, "rounds": 20, "words": list(struct.unpack("<16I", bytes.fromhex(k1)))},
        {"key": [0] * 8, "counter": 1, "rounds": 20, "words": list(struct.unpack("<16I", bytes.fromhex(k2)))},
    ]


def dense_fixture(name: str, text: str) -> dict:
    v = numpy_sim.run_text(text)
    nz = np.flatnonzero(np.abs(v) > 0)
    return {
        "name": name,
        "text": text,
        "n": int(round(np.log2(v.size))),
        "indices": [int(i) for i in nz],
        "amplitudes": [[float(v[i].real), float(v[i].imag)] for i in nz],
    }


def main() -> None:
    from oracle import oracle as O  # the seeded workload texts

    fixtures = [
        dense_fixture("clifford_t_backends_rs_18", CLIFFORD_T),
        dense_fixture("ghz_vector_rs_582", GHZ),
        dense_fixture("non_clifford_vector_rs_637", NON_CLIFFORD),
        dense_fixture("misc_named_gates", MISC),
        dense_fixture("random_layers_n8_d10_s3", O.random_circuit_text(8, 10, 3)),
        dense_fixture("reversible_n10_g60_s4", O.reversible_circuit_text(10, 60, 4)),
    ]
    out = {"chacha20": chacha_vectors(), "circuits": fixtures}
    path = os.path.join(HERE, "golden.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=0)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
