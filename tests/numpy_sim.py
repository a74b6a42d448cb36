"""An independent numpy statevector simulator (test infrastructure).

It shares no code with the C++ oracle or the CUDA engine: gate matrices are
written from their definitions and applied with ``np.tensordot`` on the
``(2,)*n`` view of the register.  It cross-checks the oracle on small
registers and generates the golden fixtures under ``tests/golden/``.

Conventions follow ncsim: qubit ``q`` is bit ``q`` of the basis index
(``src/state/vector.rs:14``); a k-qubit gate matrix is row-major over the local
index whose bit ``j`` is ``qubits[j]`` (controls first, ``src/gate.rs:316``).
"""
from __future__ import annotations

import math

import numpy as np

SQ2 = math.sqrt(2.0)


def _phase_gate(k: int, bits: int) -> np.ndarray:
    return np.diag([1.0, np.exp(2j * np.pi * k / (1 << bits))])


def named_matrix(name: str, args: list[str]) -> np.ndarray:
    n = name.upper()
    if n == "I":
        return np.eye(2, dtype=complex)
    if n == "X":
        return np.array([[0, 1], [1, 0]], dtype=complex)
    if n == "Y":
        return np.array([[0, -1j], [1j, 0]], dtype=complex)
    if n == "Z":
        return np.diag([1.0, -1.0]).astype(complex)
    if n == "H":
        return np.array([[1, 1], [1, -1]], dtype=complex) / SQ2
    if n == "S":
        return np.diag([1.0, 1j])
    if n == "S_DAG":
        return np.diag([1.0, -1j])
    if n == "T":
        return np.diag([1.0, np.exp(1j * np.pi / 4)])
    if n == "T_DAG":
        return np.diag([1.0, np.exp(-1j * np.pi / 4)])
    if n == "SQRT_X":
        return 0.5 * np.array([[1 + 1j, 1 - 1j], [1 - 1j, 1 + 1j]])
    if n == "SQRT_X_DAG":
        return 0.5 * np.array([[1 - 1j, 1 + 1j], [1 + 1j, 1 - 1j]])
    if n == "SQRT_Y":
        return 0.5 * np.array([[1 + 1j, -1 - 1j], [1 + 1j, 1 + 1j]])
    if n == "SQRT_Y_DAG":
        return 0.5 * np.array([[1 - 1j, 1 - 1j], [-1 + 1j, 1 - 1j]])
    if n in ("RX", "RY", "RZ"):
        t = float(args[0])
        c, s = math.cos(t / 2), math.sin(t / 2)
        if n == "RX":
            return np.array([[c, -1j * s], [-1j * s, c]])
        if n == "RY":
            return np.array([[c, -s], [s, c]], dtype=complex)
        return np.diag([np.exp(-0.5j * t), np.exp(0.5j * t)])
    if n == "PHASE":
        return _phase_gate(int(args[0]), int(args[1]))
    # two- and three-qubit gates: local index x = b0 + 2 b1 (+ 4 b2), controls first
    if n in ("CX", "CNOT", "CY", "CZ", "CS", "CS_DAG", "CPHASE", "SWAP"):
        m = np.zeros((4, 4), dtype=complex)
        for x in range(4):
            c, t = x & 1, x >> 1
            if n == "SWAP":
                m[t | (c << 1), x] = 1
            elif n in ("CX", "CNOT"):
                m[c | ((t ^ c) << 1), x] = 1
            elif n == "CY":
                if c:
                    m[c | ((1 - t) << 1), x] = 1j if t == 0 else -1j
                else:
                    m[x, x] = 1
            else:
                ph = {"CZ": -1.0, "CS": 1j, "CS_DAG": -1j}.get(n)
                if n == "CPHASE":
                    ph = np.exp(2j * np.pi * int(args[0]) / (1 << int(args[1])))
                m[x, x] = ph if (c and t) else 1
        return m
    if n in ("CCX", "TOFFOLI", "CCZ"):
        m = np.zeros((8, 8), dtype=complex)
        for x in range(8):
            if n == "CCZ":
                m[x, x] = -1 if x == 7 else 1
            else:
                m[x ^ 4 if (x & 3) == 3 else x, x] = 1
        return m
    raise ValueError(f"numpy_sim: unknown gate {name}")


def _poly_eval(nv: int, parts: list[str], xs: np.ndarray) -> tuple[np.ndarray, int]:
    """f(x) mod 2^bits for local values xs (uint64 array) of `bits;const;c:m,..;...`."""
    bits = int(parts[0])
    f = np.full(xs.shape, int(parts[1]) % (1 << bits), dtype=np.int64)
    for term in parts[2:]:
        c, masks = term.split(":")
        prod = np.ones(xs.shape, dtype=np.int64)
        for m in masks.split(","):
            m = np.uint64(int(m) & ((1 << nv) - 1))
            par = np.zeros(xs.shape, dtype=np.int64)
            v = xs & m
            while np.any(v):
                par ^= (v & np.uint64(1)).astype(np.int64)
                v = v >> np.uint64(1)
            prod &= par
        f = (f + int(c) * prod) % (1 << bits)
    return f, bits


def _gf2_dot(rows: list[int], x: int) -> int:
    y = 0
    for i, r in enumerate(rows):
        y |= (bin(r & x).count("1") & 1) << i
    return y


class NumpyState:
    def __init__(self, n: int):
        self.n = n
        self.v = np.zeros(1 << n, dtype=complex)
        self.v[0] = 1.0

    def apply(self, m: np.ndarray, qubits: list[int]) -> None:
        n, k = self.n, len(qubits)
        t = self.v.reshape((2,) * n)
        mt = m.reshape((2,) * (2 * k))
        col_axes = [k + (k - 1 - j) for j in range(k)]
        st_axes = [n - 1 - qubits[j] for j in range(k)]
        out = np.tensordot(mt, t, axes=(col_axes, st_axes))
        # out axes: row axes (local bit k-1 .. 0), then the untouched state axes in order
        src = list(range(k))
        dst = [n - 1 - qubits[k - 1 - a] for a in range(k)]
        self.v = np.moveaxis(out, src, dst).reshape(-1)

    def local(self, qubits: list[int]) -> np.ndarray:
        idx = np.arange(1 << self.n, dtype=np.uint64)
        x = np.zeros_like(idx)
        for j, q in enumerate(qubits):
            x |= ((idx >> np.uint64(q)) & np.uint64(1)) << np.uint64(j)
        return x

    def apply_line(self, name: str, args: list[str], qubits: list[int], raw_args: str = "") -> None:
        n = name.upper()
        if n == "DIAG":
            parts = raw_args.split(";")
            f, bits = _poly_eval(len(qubits), parts, self.local(qubits))
            self.v = self.v * np.exp(2j * np.pi * f / (1 << bits))
            return
        if n == "MONOMIAL":
            parts = raw_args.split(";")
            k = len(qubits)
            rows = [int(r) for r in parts[0].split(",")]
            shift = int(parts[1])
            s2, sp, sb = (int(a) for a in parts[-1].split(","))
            xs = np.arange(1 << k, dtype=np.uint64)
            f, bits = _poly_eval(k, parts[2:-1], xs)
            scal = (SQ2 ** s2) * np.exp(2j * np.pi * sp / (1 << sb))
            m = np.zeros((1 << k, 1 << k), dtype=complex)
            for x in range(1 << k):
                m[_gf2_dot(rows, x) ^ shift, x] = scal * np.exp(2j * np.pi * f[x] / (1 << bits))
            self.apply(m, qubits)
            return
        m = named_matrix(n, args)
        k = int(round(math.log2(m.shape[0])))
        for i in range(0, len(qubits), k):
            self.apply(m, qubits[i : i + k])


def run_text(text: str) -> np.ndarray:
    """Amplitudes after a gates-only circuit in ncsim's text format."""
    lines = []
    n = 0
    declared = None
    for raw in text.splitlines():
        line = raw.split("#")[0].strip()
        if not line:
            continue
        toks = line.split()
        if toks[0].upper() == "QUBITS":
            declared = int(toks[1])
            continue
        head = toks[0]
        if "(" in head:
            name = head[: head.index("(")]
            raw_args = head[head.index("(") + 1 : head.rindex(")")]
            args = [a.strip() for a in raw_args.split(",")]
        else:
            name, raw_args, args = head, "", []
        if name.upper() in ("TICK",):
            continue
        qs = [int(t) for t in toks[1:]]
        n = max([n] + [q + 1 for q in qs])
        lines.append((name, args, qs, raw_args))
    s = NumpyState(declared if declared is not None else n)
    for name, args, qs, raw_args in lines:
        s.apply_line(name, args, qs, raw_args)
    return s.v


def pauli_matrix_action(v: np.ndarray, n: int, x: int, z: int, phase: int) -> np.ndarray:
    """(P v) for P = i^phase X^x Z^z (ncsim's stored form, ``src/pauli/ops.rs:5``)."""
    idx = np.arange(1 << n, dtype=np.uint64)
    # P|c> = i^{phase + 2 popcount(z & c)} |c ^ x>
    pc = np.zeros(idx.shape, dtype=np.int64)
    t = idx & np.uint64(z)
    while np.any(t):
        pc += (t & np.uint64(1)).astype(np.int64)
        t = t >> np.uint64(1)
    ph = (1j) ** ((phase + 2 * pc) % 4)
    out = np.zeros_like(v)
    out[(idx ^ np.uint64(x)).astype(np.int64)] = ph * v
    return out
